// fluid_oracle.hpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of solunar's particle-fluid step, the checker for the CUDA library.  Only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it; the library never
// links or calls it.  Templated on the arithmetic type: `float` is the parity oracle and the
// timed CPU baseline, `double` is the precision oracle, and `DualOf<float | double>` (dual.hpp)
// carries the exact derivative of the FP32 program or of the FP64 method along one direction for
// the adjoint's checks (oracle_tangent.cpp).
//
// It follows, function by function (paths relative to the reference project):
//   src/fluid/mod.rs      Kernel :125-165, Grid :169-262, near :264-277, Lists :279-308,
//                         add_particle :412, set_domain :433, keep_in_domain :451,
//                         fill_box :493-524, cell_of :526-533, update_neighbors :540-608,
//                         compute_densities :621-675, state_hash :677-691, rest_mass :694-709
//   src/fluid/step.rs     step :58-90, fastest :92-96, wcsph :102-116, wcsph_steps :118-142,
//                         wcsph_substep :144-224, viscous :229-251, viscosity :254-259,
//                         wall_viscous :262-301, advance :305-339
//   src/fluid/dfsph.rs    dfsph :46-77, dfsph_substep :79-103, gradients :108-136,
//                         factors :138-163, density_rate :166-181, push_apart :184-216,
//                         solve :222-275
//   src/fluid/boundary.rs add_box_container :41-68, add_wall :74-91, remove_boundary :94-115,
//                         cells_in :123-126, check_room :128-137, settle_walls :155-178,
//                         check_box :230-238, union :240-247
//   src/fluid/flow.rs     CLEAR_SHARE :7, add_emitter :86-99, add_drain :104-106,
//                         remove_flow :109-113, add_flow :115-139, run_flows :144-231
//   src/fluid/terrain.rs  TerrainField read :100-136, sample :139-142, ground :144-171,
//                         GroundSites :176-245, solid :248-250, add_terrain :262-302 (the caller
//                         samples the distance field), ground_near :305-310, terrain_contact :314-333
//   src/fluid/save.rs     save_snapshot :18-73, load_snapshot :79-181 (Walls::save/load
//                         boundary.rs:182-227, Flows::save/load flow.rs:36-83)
//   src/snapshot/bytes.rs fnv1a :6-13, Writer :15-67, Reader :89-157
//
// Arithmetic follows the reference's scalar code: left-to-right evaluation, no fused
// multiply-add (build with -ffp-contract=off), IEEE division and square root, `powi` as binary
// exponentiation, `Iterator::sum` as a sequential fold.  The reference's vector type comes from
// the un-vendored `algebrix` crate (git rev 1bf888b98936f382f1def04ce06b15fbbfcdd46d); its
// operations are assumed to be componentwise IEEE f32 with dot = x*x' + y*y' + z*z' summed left
// to right, length = sqrt(dot), v / s divided per component, normalize_or dividing by the
// length.  Parity with the Rust binary itself is therefore unpinned at the bit level; the
// reference's own tests (property tests, no stored vectors) pin this restatement instead.
//
// Movers (rigid coupling) are not on the path: they are absent from this restatement, as they
// are empty in every configuration it is run on.
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include "dual.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

enum Status : int32_t {
    OK = 0,
    INVALID_SETTINGS = 1,
    NON_FINITE = 2,
    OUT_OF_RANGE = 3,
    FLUID_FULL = 4,
    DISPATCH_INCOMPLETE = 5,
    UNSUPPORTED = 6,
    INVALID_ARGUMENT = 9,
    SNAPSHOT = 10,  // SnapshotError (src/snapshot/mod.rs:56-63)
    INVALID_SHAPE = 11,  // PhysicsError::InvalidShape (src/error.rs:10)
};

// ---- scalar helpers ---------------------------------------------------------------------

// The standard functions on the restatement's scalar.  Called unqualified, so that a derivative
// number type (dual.hpp) supplies its own by argument-dependent lookup; for float and double
// they are the standard functions themselves.
template <class R> inline R osqrt(R x) { return std::sqrt(x); }
template <class R> inline R ofloor(R x) { return std::floor(x); }
template <class R> inline R oceil(R x) { return std::ceil(x); }
template <class R> inline R oround(R x) { return std::round(x); }
template <class R> inline R ofabs(R x) { return std::fabs(x); }
template <class R> inline bool oisnan(R x) { return std::isnan(x); }
template <class R> inline bool oisfinite(R x) { return std::isfinite(x); }

// Rust f32::min / f32::max: a NaN operand yields the other one.
template <class R> inline R rmin(R a, R b) {
    if (oisnan(a)) return b;
    if (oisnan(b)) return a;
    return b < a ? b : a;
}
template <class R> inline R rmax(R a, R b) {
    if (oisnan(a)) return b;
    if (oisnan(b)) return a;
    return b > a ? b : a;
}
// Rust's `f as i32`: saturating, NaN to 0
template <class R> inline int32_t as_i32(R v) {
    if (oisnan(v)) return 0;
    if (v >= R(2147483647.0)) return INT32_MAX;
    if (v <= R(-2147483648.0)) return INT32_MIN;
    return int32_t(v);
}
// f32::total_cmp's order: -NaN < -inf < ... < -0 < +0 < ... < +inf < +NaN
template <class R> inline bool total_less(R a, R b) {
    static_assert(sizeof(R) == 4 || sizeof(R) == 8, "total_less: a float or a double");
    using U = typename std::conditional<sizeof(R) == 4, int32_t, int64_t>::type;
    using UU = typename std::make_unsigned<U>::type;
    U x, y;
    std::memcpy(&x, &a, sizeof(R));
    std::memcpy(&y, &b, sizeof(R));
    const int shift = int(8 * sizeof(R) - 1);
    x ^= U(UU(x >> shift) >> 1);
    y ^= U(UU(y >> shift) >> 1);
    return x < y;
}
// `powi` lowered to binary exponentiation (mod.rs:136,145,154; step.rs:149,156).
template <class R> inline R pow2(R x) { return x * x; }
template <class R> inline R pow3(R x) { return x * (x * x); }
template <class R> inline R pow4(R x) { R s = x * x; return s * s; }
template <class R> inline R pow7(R x) { R s = x * x; R q = s * s; return (x * s) * q; }

// Rust `as i32` from a float: saturating, NaN to zero (mod.rs:529-531).
template <class R> inline int32_t sat_i32(R v) {
    if (oisnan(v)) return 0;
    if (v >= R(2147483647.0)) return std::numeric_limits<int32_t>::max();
    if (v <= R(-2147483648.0)) return std::numeric_limits<int32_t>::min();
    return static_cast<int32_t>(v);
}

template <class R> inline uint64_t bits_of(R v) {
    static_assert(sizeof(R) == 4 || sizeof(R) == 8, "bits_of: a float or a double");
    if constexpr (std::is_same_v<R, float>) {
        uint32_t b;
        std::memcpy(&b, &v, 4);
        return b;
    } else {
        uint64_t b;
        std::memcpy(&b, &v, 8);
        return b;
    }
}

// ---- vectors ------------------------------------------------------------------------------

template <class R> struct V3 {
    R x{0}, y{0}, z{0};
    V3() = default;
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    static V3 splat(R v) { return V3(v, v, v); }
    bool operator==(const V3& o) const { return x == o.x && y == o.y && z == o.z; }
    bool operator!=(const V3& o) const { return !(*this == o); }
};
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> operator/(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline R length_squared(V3<R> a) { return dot(a, a); }
template <class R> inline R length(V3<R> a) { return osqrt(length_squared(a)); }
template <class R> inline bool is_finite(V3<R> a) {
    return oisfinite(a.x) && oisfinite(a.y) && oisfinite(a.z);
}
template <class R> inline V3<R> vmin(V3<R> a, V3<R> b) { return {rmin(a.x, b.x), rmin(a.y, b.y), rmin(a.z, b.z)}; }
template <class R> inline V3<R> vmax(V3<R> a, V3<R> b) { return {rmax(a.x, b.x), rmax(a.y, b.y), rmax(a.z, b.z)}; }
template <class R> inline V3<R> clamp(V3<R> v, V3<R> lo, V3<R> hi) { return vmin(vmax(v, lo), hi); }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
// q * v for the unit quaternion (x, y, z, w): v (w^2 - |b|^2) + b 2 (v.b) + (b x v) 2 w, b = (x, y, z)
template <class R> inline V3<R> rotate(const R q[4], V3<R> v) {
    V3<R> b(q[0], q[1], q[2]);
    R w = q[3];
    R b2 = dot(b, b);
    return v * (w * w - b2) + b * (dot(v, b) * R(2)) + cross(b, v) * (w * R(2));
}
template <class R> inline V3<R> normalize_or(V3<R> v, V3<R> fallback) {
    R len = length(v);
    if (oisfinite(len) && len > R(0)) return v / len;
    return fallback;
}

// ---- settings -------------------------------------------------------------------------------

struct Settings {
    int32_t solver = 0;  // 0 WCSPH, 1 DFSPH
    float spacing = 0.05f;
    float rest_density = 1000.0f;
    float support = 2.0f;
    uint64_t max_particles = uint64_t(1) << 22;
    float sound_speed = 20.0f;
    float viscosity = 0.15f;
    float gravity[3] = {0.0f, -9.81f, 0.0f};
    float courant = 0.4f;
    uint32_t max_substeps = 2000;
    float divergence_tolerance = 1e-3f;
    float density_tolerance = 5e-4f;
    uint32_t min_iterations = 2;
    uint32_t max_iterations = 100;
    // 0: the reference's sequential sum of the solver error in the working precision
    //    (dfsph.rs:266-267); 1: a compensated sum in double, as the CUDA library takes it.
    int32_t residual_sum = 0;
    // 1: each DFSPH solve starts with one push at half the stiffness impulse (sum of kappa dt)
    //    the particle's solve of the same kind applied the substep before.  The reference
    //    cold-starts every solve, because a half-pressure start pushed water apart and sped a
    //    dam-break front up (dfsph.rs:217-221): 0, the default.
    int32_t warm_start = 0;

    // mod.rs:98-117
    bool valid() const {
        auto positive = [](float v) { return oisfinite(v) && v > 0.0f; };
        bool support_ok = support >= 1.5f && support <= 4.0f;
        return positive(spacing) && positive(rest_density) && support_ok && max_particles > 0 &&
               positive(sound_speed) && oisfinite(viscosity) && viscosity >= 0.0f &&
               oisfinite(gravity[0]) && oisfinite(gravity[1]) && oisfinite(gravity[2]) &&
               courant > 0.0f && courant <= 1.0f && max_substeps > 0;
    }
};

struct Report {
    uint32_t substeps = 0;
    int32_t capped = 0;
    float max_compression = 0;
    float max_speed = 0;
    uint32_t held_back = 0;
    uint32_t iterations = 0;
    uint32_t emitted = 0, drained = 0, lost = 0;
    float sound_speed = 0;
};

// ---- kernel (mod.rs:125-165) ------------------------------------------------------------

template <class R> struct Kernel {
    R radius{0}, scale{0};
    Kernel() = default;
    explicit Kernel(R r) : radius(r), scale(R(21) / (R(2) * R(3.14159265358979323846) * pow3(r))) {}
    R value(R distance) const {
        R q = distance / radius;
        if (q >= R(1)) return R(0);
        return scale * pow4(R(1) - q) * (R(1) + R(4) * q);
    }
    R slope(R distance) const {
        R q = distance / radius;
        if (q >= R(1)) return R(0);
        return scale * R(-20) * q * pow3(R(1) - q) / radius;
    }
    V3<R> gradient(V3<R> offset) const {
        R distance = length(offset);
        if (distance <= R(0)) return V3<R>();
        return offset * (slope(distance) / distance);
    }
};

// ---- grid (mod.rs:167-262) -----------------------------------------------------------------

struct Key {
    int32_t x, y, z;
    bool operator==(const Key& o) const { return x == o.x && y == o.y && z == o.z; }
    bool operator!=(const Key& o) const { return !(*this == o); }
    bool operator<(const Key& o) const { return std::tie(x, y, z) < std::tie(o.x, o.y, o.z); }
};

struct Range {
    uint32_t begin, end;
    bool operator==(const Range& o) const { return begin == o.begin && end == o.end; }
};

struct Grid {
    std::vector<std::pair<Key, Range>> cells;
    std::vector<uint32_t> dense;
    Key low{0, 0, 0};
    int64_t span[3] = {0, 0, 0};

    // `keys` already sorted (mod.rs:182-197).
    static Grid build(const std::vector<Key>& keys) {
        Grid g;
        for (size_t i = 0; i < keys.size(); ++i) {
            uint32_t index = uint32_t(i);
            if (!g.cells.empty() && g.cells.back().first == keys[i]) {
                g.cells.back().second.end = index + 1;
            } else {
                g.cells.push_back({keys[i], Range{index, index + 1}});
            }
        }
        g.index();
        return g;
    }

    // mod.rs:199-227: a dense table while its box is at most 64 cells per occupied one + 4096.
    void index() {
        if (cells.empty()) return;
        Key lo = cells[0].first, hi = cells[0].first;
        for (auto& c : cells) {
            lo = Key{std::min(lo.x, c.first.x), std::min(lo.y, c.first.y), std::min(lo.z, c.first.z)};
            hi = Key{std::max(hi.x, c.first.x), std::max(hi.y, c.first.y), std::max(hi.z, c.first.z)};
        }
        int64_t sx = int64_t(hi.x) - lo.x + 1, sy = int64_t(hi.y) - lo.y + 1, sz = int64_t(hi.z) - lo.z + 1;
        // saturating products, as i64::saturating_mul
        auto sat_mul = [](int64_t a, int64_t b) -> int64_t {
            __int128 p = (__int128)a * b;
            if (p > std::numeric_limits<int64_t>::max()) return std::numeric_limits<int64_t>::max();
            return (int64_t)p;
        };
        int64_t volume = sat_mul(sat_mul(sx, sy), sz);
        if (volume > 64 * int64_t(cells.size()) + 4096) return;
        dense.assign(size_t(volume), UINT32_MAX);
        for (size_t slot = 0; slot < cells.size(); ++slot) {
            const Key& c = cells[slot].first;
            int64_t at = (int64_t(c.x - lo.x) * sy + int64_t(c.y - lo.y)) * sz + int64_t(c.z - lo.z);
            dense[size_t(at)] = uint32_t(slot);
        }
        low = lo;
        span[0] = sx;
        span[1] = sy;
        span[2] = sz;
    }

    bool range(Key key, Range& out) const {
        size_t slot;
        if (dense.empty()) {
            auto it = std::lower_bound(cells.begin(), cells.end(), key,
                                       [](const std::pair<Key, Range>& c, const Key& k) { return c.first < k; });
            if (it == cells.end() || it->first != key) return false;
            slot = size_t(it - cells.begin());
        } else {
            int64_t x = int64_t(key.x) - low.x, y = int64_t(key.y) - low.y, z = int64_t(key.z) - low.z;
            if (x < 0 || x >= span[0] || y < 0 || y >= span[1] || z < 0 || z >= span[2]) return false;
            uint32_t s = dense[size_t((x * span[1] + y) * span[2] + z)];
            if (s == UINT32_MAX) return false;
            slot = s;
        }
        out = cells[slot].second;
        return true;
    }

    // The 27 cells around, dz outer, then dy, dx inner (mod.rs:250-261).  Neighbour keys are
    // formed in 64-bit; one past the i32 range holds nothing.
    void around(Key c, std::vector<Range>& out) const {
        out.clear();
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int64_t x = int64_t(c.x) + dx, y = int64_t(c.y) + dy, z = int64_t(c.z) + dz;
                    if (x > INT32_MAX || x < INT32_MIN || y > INT32_MAX || y < INT32_MIN || z > INT32_MAX ||
                        z < INT32_MIN)
                        continue;
                    Range r;
                    if (range(Key{int32_t(x), int32_t(y), int32_t(z)}, r)) out.push_back(r);
                }
    }
};

// CSR neighbour lists (mod.rs:279-308).
struct Lists {
    std::vector<uint32_t> start;
    std::vector<uint32_t> items;
    size_t count(size_t i) const {
        if (i + 1 >= start.size()) return 0;
        return start[i + 1] - start[i];
    }
};

inline uint64_t fnv1a(const uint8_t* data, size_t n) {
    uint64_t hash = 0xcbf29ce484222325ull;
    for (size_t i = 0; i < n; ++i) {
        hash ^= uint64_t(data[i]);
        hash *= 0x00000100000001b3ull;
    }
    return hash;
}

// Compensated sum in double (Neumaier), the CUDA library's residual reduction.
struct CompensatedSum {
    double sum = 0.0, carry = 0.0;
    void add(double v) {
        double t = sum + v;
        if (ofabs(sum) >= ofabs(v)) carry += (sum - t) + v;
        else carry += (v - t) + sum;
        sum = t;
    }
    double value() const { return sum + carry; }
};

// ---- walls (boundary.rs:20-33) ------------------------------------------------------------

template <class R> struct Container {
    uint32_t id;
    V3<R> low, high;
};

template <class R> struct Walls {
    std::vector<V3<R>> positions;
    std::vector<uint32_t> owners;
    Grid grid;
    uint32_t next = 0;
    bool has_bounds = false;
    V3<R> bounds_low, bounds_high;
    std::vector<Container<R>> containers;
};

// ---- the world --------------------------------------------------------------------------------

template <class R> class World {
  public:
    using Vec = V3<R>;

    Settings settings;
    Kernel<R> kernel;
    R mass{0};
    std::vector<uint32_t> ids;
    std::vector<Vec> positions, velocities;
    std::vector<R> densities;
    // warm starts: per particle the stiffness impulse its last divergence (0) and density (1)
    // solve applied, kept in particle order like the densities
    std::vector<R> impulse[2];
    uint32_t next_id = 0;
    Grid grid;
    Lists neighbors, wall_neighbors, mover_neighbors;
    Walls<R> walls;
    bool has_domain = false;
    Vec domain_low, domain_high;
    // emitters and drains (flow.rs:14-33), in the order they were added
    struct Flow {
        uint32_t id;
        Vec low, high;
        bool emitter;
        Vec velocity;
    };
    std::vector<Flow> flows;
    uint32_t flow_next = 0;
    // terrain regions (terrain.rs:36-42) and what ground does to a particle (terrain.rs:176-186)
    struct Terrain {
        uint32_t owner;
        Vec low;
        size_t nx, ny, nz;
        R step;
        std::vector<R> distances;
    };
    std::vector<Terrain> terrains;
    struct GroundSites {
        R spacing{0}, reach{0}, low{0}, step{0};
        std::vector<Vec> offsets;
        std::vector<R> weights, fars, damping;
    } sites;
    std::vector<Vec> ground_slopes;  // mod.rs:320-322: empty without terrains
    // coupled bodies (couple.rs:15-33), in body order, and their points for the running step
    // (couple.rs:35-47)
    struct Coupled {
        uint64_t body;  // BodyHandle (index, generation) as index << 32 | generation
        std::vector<Vec> points, probes;
        R probe_spacing{0};
        Vec center, velocity, moved;
        Vec impulse, angular;  // what the water's damping did to the body this step
    };
    std::vector<Coupled> coupled;
    struct Movers {
        std::vector<Vec> start, positions, velocities;
        std::vector<uint32_t> owners;
        Grid grid;
    } movers;
    // per-pair gradient caches of the last DFSPH substep (dfsph.rs:24-41)
    std::vector<Vec> grad_fluid, grad_walls;
    // solver iteration counts of the last DFSPH substep: divergence, density
    uint32_t last_iterations[2] = {0, 0};
    // Iteration counts the next solves take regardless of their errors (divergence, density of
    // each substep in turn): a derivative run then differentiates the same discrete steps as the
    // run it checks.  Empty (the default): solves stop on their tolerances.
    std::vector<uint32_t> forced_iterations;
    size_t forced_next = 0;
    // A derivative run only: quantities held constant (their derivative dropped), to measure
    // what each path of the DFSPH substep contributes to a tangent.  Bits: 1 fluid pair
    // gradients, 2 wall pair gradients, 4 factors, 8 densities, 16 viscosity and gravity's
    // velocity change, 32 solver stiffnesses, 64 the fluid pairs' viscosity, 128 the walls'.
    uint32_t hold = 0;
    template <class T> T constant_if(T x, uint32_t bit) const {
        if constexpr (is_dual<R>::value) {
            if (hold & bit) {
                if constexpr (std::is_same<T, Vec>::value) return Vec(R(double(x.x)), R(double(x.y)), R(double(x.z)));
                else return R::of(x.v, 0.0);
            }
        }
        return x;
    }
    int threads = 0;  // 0: OpenMP default

    static Status create(const Settings& s, World& out) {
        if (!s.valid()) return INVALID_SETTINGS;
        out = World();
        out.settings = s;
        out.kernel = Kernel<R>(radius_of(s));
        out.mass = rest_mass(s);
        out.build_ground_sites();
        return OK;
    }

    static constexpr size_t kMaxTerrainNodes = size_t(1) << 24;  // terrain.rs:9
    static constexpr int kMapSamples = 256;                      // terrain.rs:11

    // GroundSites::new (terrain.rs:188-238)
    void build_ground_sites() {
        const R spacing = R(settings.spacing), r = radius();
        GroundSites g;
        g.spacing = spacing;
        int reach = int(oceil(r / spacing));
        for (int z = -reach; z <= reach; ++z)
            for (int y = -reach; y <= reach; ++y)
                for (int x = -reach; x <= reach; ++x) {
                    Vec offset = Vec(R(x), R(y), R(z)) * spacing;
                    R far = length(offset);
                    if (far < r) {
                        g.offsets.push_back(offset);
                        g.weights.push_back(mass * kernel.value(far));
                        g.fars.push_back(far);
                    }
                }
        g.low = -spacing / R(2);
        g.step = (r - g.low) / R(kMapSamples - 1);
        R soften = R(0.01f) * r * r;
        int across_reach = reach + 1;
        for (int sample = 0; sample < kMapSamples; ++sample) {
            R distance = g.low + g.step * R(sample);
            R weight = R(0);
            for (int layer = 0;; ++layer) {
                R depth = distance + spacing * (R(layer) + R(0.5));
                if (depth >= r) break;
                for (int a = -across_reach; a <= across_reach; ++a)
                    for (int b = -across_reach; b <= across_reach; ++b) {
                        R across = R(a * a + b * b) * spacing * spacing;
                        R squared = across + depth * depth;
                        R far = osqrt(squared);
                        if (far >= r || far <= R(0)) continue;
                        weight += mass * depth * depth * -kernel.slope(far) / (far * (squared + soften));
                    }
            }
            g.damping.push_back(weight);
        }
        g.reach = r + spacing / R(2);
        sites = std::move(g);
    }

    // GroundSites::damping (terrain.rs:241-249)
    R damping(R distance) const {
        R at = (rmax(distance, sites.low) - sites.low) / sites.step;
        size_t below = size_t(ofloor(at));
        if (below + 1 >= size_t(kMapSamples)) return R(0);
        R part = at - R(below);
        return sites.damping[below] + (sites.damping[below + 1] - sites.damping[below]) * part;
    }

    // TerrainField::read (terrain.rs:100-136): trilinear value and its change per axis
    bool terrain_read(const Terrain& t, Vec point, R& value, Vec& change) const {
        Vec local = (point - t.low) / t.step;
        auto inside = [](R v, size_t nodes) { return v >= R(0) && v <= R(nodes - 1); };
        if (!(inside(local.x, t.nx) && inside(local.y, t.ny) && inside(local.z, t.nz))) return false;
        auto base = [](R v, size_t nodes) { return std::min(size_t(ofloor(v)), nodes - 2); };
        size_t x = base(local.x, t.nx), y = base(local.y, t.ny), z = base(local.z, t.nz);
        R fx = local.x - R(x), fy = local.y - R(y), fz = local.z - R(z);
        auto corner = [&](size_t dx, size_t dy, size_t dz) {
            return t.distances[((y + dy) * t.nz + (z + dz)) * t.nx + (x + dx)];
        };
        auto lerp = [](R a, R b, R u) { return a + (b - a) * u; };
        auto face = [&](size_t dy, size_t dz, R& v, R& g) {
            R a = corner(0, dy, dz), b = corner(1, dy, dz);
            v = lerp(a, b, fx);
            g = b - a;
        };
        R v00, g00, v10, g10, v01, g01, v11, g11;
        face(0, 0, v00, g00);
        face(1, 0, v10, g10);
        face(0, 1, v01, g01);
        face(1, 1, v11, g11);
        R v0 = lerp(v00, v10, fy), v1 = lerp(v01, v11, fy);
        value = lerp(v0, v1, fz);
        change = Vec(lerp(lerp(g00, g10, fy), lerp(g01, g11, fy), fz), lerp(v10 - v00, v11 - v01, fz), v1 - v0) / t.step;
        return true;
    }

    // TerrainField::sample (terrain.rs:139-142)
    bool terrain_sample(const Terrain& t, Vec point, R& distance, Vec& normal) const {
        Vec change;
        if (!terrain_read(t, point, distance, change)) return false;
        normal = normalize_or(change, Vec(R(0), R(1), R(0)));
        return true;
    }

    // solid (terrain.rs:248-250)
    static R solid(R distance, R size) {
        R v = R(0.5) - distance / size;
        return v < R(0) ? R(0) : (v > R(1) ? R(1) : v);
    }

    // TerrainField::ground (terrain.rs:144-171): false outside the region
    bool terrain_ground(const Terrain& t, Vec point, R& distance, Vec& normal, R& density, Vec& gradient) const {
        Vec change;
        if (!terrain_read(t, point, distance, change)) return false;
        density = R(0);
        gradient = Vec();
        if (distance < sites.reach) {
            R open = distance - sites.spacing / R(2);
            for (size_t k = 0; k < sites.offsets.size(); ++k) {
                if (sites.fars[k] <= open) continue;
                R there;
                Vec toward;
                if (!terrain_read(t, point + sites.offsets[k], there, toward)) continue;
                R share = solid(there, sites.spacing);
                density += sites.weights[k] * share;
                if (share > R(0) && share < R(1)) gradient = gradient - toward * (sites.weights[k] / sites.spacing);
            }
        }
        normal = normalize_or(change, Vec(R(0), R(1), R(0)));
        return true;
    }

    // terrain_contact (terrain.rs:314-333): true when the particle got under a surface
    bool terrain_contact(R rest, Vec& at, Vec& velocity) const {
        bool under = false;
        for (const Terrain& t : terrains) {
            R distance;
            Vec normal;
            if (!terrain_sample(t, at, distance, normal)) continue;
            if (distance < rest) {
                under = under || distance < R(0);
                at = at + normal * (rest - distance);
                R into = dot(velocity, normal);
                if (into < R(0)) velocity = velocity - normal * into;
            }
        }
        return under;
    }

    // add_terrain's node lattice (terrain.rs:275-283): step spacing/2, nodes per axis
    Status terrain_nodes(Vec low, Vec high, size_t nodes[3]) const {
        if (!is_finite(low) || !is_finite(high)) return NON_FINITE;
        if (high.x <= low.x || high.y <= low.y || high.z <= low.z) return OUT_OF_RANGE;
        R step = R(settings.spacing) / R(2);
        auto count = [&](R extent) { return size_t(rmin(oceil(extent / step), R(1e7))) + 1; };
        Vec size = high - low;
        nodes[0] = count(size.x);
        nodes[1] = count(size.y);
        nodes[2] = count(size.z);
        unsigned __int128 total = (unsigned __int128)nodes[0] * nodes[1] * nodes[2];
        if (total > kMaxTerrainNodes) return FLUID_FULL;
        return OK;
    }

    // add_terrain (terrain.rs:262-302) with the distances the caller sampled at the nodes
    // low + (x, y, z) spacing/2, in (y, z, x) order, x fastest
    Status add_terrain(Vec low, Vec high, const float* distances, size_t count, uint32_t* id_out) {
        size_t nodes[3];
        Status st = terrain_nodes(low, high, nodes);
        if (st != OK) return st;
        if (count != nodes[0] * nodes[1] * nodes[2]) return INVALID_ARGUMENT;
        Terrain t;
        t.low = low;
        t.nx = nodes[0];
        t.ny = nodes[1];
        t.nz = nodes[2];
        t.step = R(settings.spacing) / R(2);
        t.distances.assign(distances, distances + count);
        t.owner = add_wall_points({});
        terrains.push_back(std::move(t));
        if (id_out) *id_out = terrains.back().owner;
        return OK;
    }

    static R radius_of(const Settings& s) { return R(s.spacing) * R(s.support); }
    R radius() const { return radius_of(settings); }
    size_t len() const { return ids.size(); }
    Vec gravity() const { return Vec(param(settings.gravity[0], 2), param(settings.gravity[1], 3), param(settings.gravity[2], 4)); }
    // A physics parameter as the step reads it: its value, and for a derivative run (R = DualOf)
    // the tangent seeded for it (0 viscosity, 1 sound speed, 2-4 gravity).
    double param_tangent[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    R param(float v, int which) const {
        if constexpr (is_dual<R>::value) return R(double(v), param_tangent[which]);
        else return R(v);
    }

    // mod.rs:694-709
    static R rest_mass(const Settings& s) {
        Kernel<R> k(radius_of(s));
        int reach = int(oceil(s.support));
        R sum = R(0);
        for (int z = -reach; z <= reach; ++z)
            for (int y = -reach; y <= reach; ++y)
                for (int x = -reach; x <= reach; ++x) {
                    Vec offset = Vec(R(x), R(y), R(z)) * R(s.spacing);
                    sum += k.value(length(offset));
                }
        return R(s.rest_density) / sum;
    }

    // mod.rs:412-426
    Status add_particle(Vec position, Vec velocity, uint32_t* id_out) {
        if (!is_finite(position) || !is_finite(velocity)) return NON_FINITE;
        if (len() >= settings.max_particles || next_id == UINT32_MAX) return FLUID_FULL;
        uint32_t id = next_id++;
        ids.push_back(id);
        positions.push_back(position);
        velocities.push_back(velocity);
        densities.push_back(R(0));
        impulse[0].push_back(R(0));
        impulse[1].push_back(R(0));
        if (id_out) *id_out = id;
        return OK;
    }

    // mod.rs:433-444
    Status set_domain(const Vec* low, const Vec* high) {
        if (low && high) {
            if (!is_finite(*low) || !is_finite(*high)) return NON_FINITE;
            if (high->x <= low->x || high->y <= low->y || high->z <= low->z) return OUT_OF_RANGE;
            has_domain = true;
            domain_low = *low;
            domain_high = *high;
        } else {
            has_domain = false;
        }
        return OK;
    }

    // mod.rs:451-486
    uint32_t keep_in_domain() {
        if (!has_domain) return 0;
        size_t kept = 0;
        uint32_t lost = 0;
        for (size_t i = 0; i < len(); ++i) {
            if (clamp(positions[i], domain_low, domain_high) == positions[i]) {
                ids[kept] = ids[i];
                positions[kept] = positions[i];
                velocities[kept] = velocities[i];
                densities[kept] = densities[i];
                impulse[0][kept] = impulse[0][i];
                impulse[1][kept] = impulse[1][i];
                ++kept;
            } else {
                ++lost;
            }
        }
        ids.resize(kept);
        positions.resize(kept);
        velocities.resize(kept);
        densities.resize(kept);
        impulse[0].resize(kept);
        impulse[1].resize(kept);
        return lost;
    }

    // flow.rs:115-139
    Status add_flow(Vec low, Vec high, bool emitter, Vec velocity, uint32_t* id_out) {
        if (!is_finite(low) || !is_finite(high)) return NON_FINITE;
        if (high.x <= low.x || high.y <= low.y || high.z <= low.z) return OUT_OF_RANGE;
        if (flow_next == UINT32_MAX) return FLUID_FULL;
        uint32_t id = flow_next++;
        flows.push_back(Flow{id, low, high, emitter, velocity});
        if (id_out) *id_out = id;
        return OK;
    }

    // flow.rs:86-99, 104-106
    Status add_emitter(Vec low, Vec high, Vec velocity, uint32_t* id_out) {
        if (!is_finite(velocity)) return NON_FINITE;
        return add_flow(low, high, true, velocity, id_out);
    }
    Status add_drain(Vec low, Vec high, uint32_t* id_out) { return add_flow(low, high, false, Vec(), id_out); }

    // ---- coupled bodies (src/fluid/couple.rs, lift.rs) -------------------------------------

    // A body's place and motion for a step (substep.rs SubstepPose, as couple.rs:418-426 reads
    // it): position in f64 as the rigid world keeps it, rotation (x, y, z, w), velocities;
    // `dynamic` when the body takes pushes (a fixed or kinematic one refuses them).
    struct Pose {
        uint64_t body;
        double position[3];
        float rotation[4];
        float linear[3], angular[3];
        int32_t dynamic;
    };
    // What the water did to a body over a step: lift.rs's lift (given back to the water when the
    // body is dynamic) and the damping impulse of couple.rs:375-416.
    struct Push {
        uint64_t body;
        Vec lift, lift_angular, damping, damping_angular;
        int32_t lifted;
    };
    static constexpr size_t kMaxProbes = 4096;  // lift.rs:8

    // couple.rs:453-511: lattice points `spacing` apart inside the shape (0 cuboid with half
    // extents, 1 sphere with radius, 2 capsule with radius and half height), no deeper than
    // `reach`, centred on it; FLUID_FULL past `limit` points
    static Status shape_points(int kind, const float dims[3], R spacing, R reach, size_t limit, std::vector<Vec>& out) {
        out.clear();
        Vec half;
        R a = R(dims[0]), b = R(dims[1]), c = R(dims[2]);
        if (kind == 0) {
            half = Vec(a, b, c);
        } else if (kind == 1) {
            half = Vec::splat(a);
        } else if (kind == 2) {
            if (!(b >= R(0))) return INVALID_SHAPE;  // a capsule's half height is not negative
            half = Vec(a, b + a, a);
        } else {
            return INVALID_SHAPE;
        }
        if (!is_finite(half) || rmin(rmin(half.x, half.y), half.z) <= R(0)) return INVALID_SHAPE;
        auto depth = [&](Vec at) -> R {
            if (kind == 0) {
                Vec room = half - Vec(ofabs(at.x), ofabs(at.y), ofabs(at.z));
                return rmin(rmin(room.x, room.y), room.z);
            }
            if (kind == 1) return a - length(at);
            R y = rmin(rmax(at.y, -b), b);
            return a - length(at - Vec(R(0), y, R(0)));
        };
        auto count = [&](R extent) -> int64_t {
            R v = ofloor(R(2) * extent / spacing);
            int64_t k = oisnan(v) ? 0 : (v >= R(4096) ? 4096 : (v <= R(0) ? 0 : int64_t(v)));
            return k;
        };
        int64_t cx = count(half.x), cy = count(half.y), cz = count(half.z);
        if (cx * cy * cz > int64_t(std::min<size_t>(limit, size_t(INT64_MAX)))) return FLUID_FULL;
        auto start = [&](int64_t cells) { return -(R(float(cells)) - R(1)) * spacing / R(2); };
        Vec origin(start(cx), start(cy), start(cz));
        for (int64_t y = 0; y < cy; ++y)
            for (int64_t z = 0; z < cz; ++z)
                for (int64_t x = 0; x < cx; ++x) {
                    Vec at = origin + Vec(R(float(x)), R(float(y)), R(float(z))) * spacing;
                    R inside = depth(at);
                    if (inside >= R(0) && inside <= reach) out.push_back(at);
                }
        return OK;
    }

    size_t coupled_points() const {
        size_t k = 0;
        for (auto& c : coupled) k += c.points.size();
        return k;
    }

    // couple.rs:165-200
    Status couple(uint64_t body, int kind, const float dims[3]) {
        std::vector<Vec> points, probes;
        Status st = shape_points(kind, dims, R(settings.spacing), radius(), size_t(settings.max_particles), points);
        if (st != OK) return st;
        if (points.empty()) return INVALID_SHAPE;
        uint64_t used = coupled_points();
        uint64_t room = settings.max_particles > used ? settings.max_particles - used : 0;
        if (points.size() > room) return FLUID_FULL;
        // coarser probes for a big body, each standing for its share of the volume
        R probe_spacing = R(settings.spacing);
        for (;;) {
            st = shape_points(kind, dims, probe_spacing, R(INFINITY), kMaxProbes, probes);
            if (st == FLUID_FULL) {
                probe_spacing = probe_spacing * R(1.25f);
                continue;
            }
            if (st != OK) return st;
            if (probes.empty()) {
                probe_spacing = R(settings.spacing);
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
        return OK;
    }

    // couple.rs:203-207
    bool uncouple(uint64_t body) {
        size_t before = coupled.size();
        coupled.erase(std::remove_if(coupled.begin(), coupled.end(), [&](const Coupled& c) { return c.body == body; }),
                      coupled.end());
        return coupled.size() != before;
    }

    static const Pose* pose_of(const Pose* poses, size_t n, uint64_t body) {
        for (size_t k = 0; k < n; ++k)
            if (poses[k].body == body) return &poses[k];
        return nullptr;
    }
    static Vec center_of(const Pose& p) {
        // position.to_dvec3().as_vec3(): the f64 position rounded to f32
        return Vec(R(float(p.position[0])), R(float(p.position[1])), R(float(p.position[2])));
    }
    static void quat_of(const Pose& p, R q[4]) {
        for (int k = 0; k < 4; ++k) q[k] = R(p.rotation[k]);
    }

    // couple.rs:255-288: body points where the poses say, bodies without a pose uncoupled
    void place_movers_at(const Pose* poses, size_t npose) {
        coupled.erase(std::remove_if(coupled.begin(), coupled.end(),
                                     [&](const Coupled& c) { return !pose_of(poses, npose, c.body); }),
                      coupled.end());
        Movers m;
        for (size_t owner = 0; owner < coupled.size(); ++owner) {
            Coupled& known = coupled[owner];
            const Pose& state = *pose_of(poses, npose, known.body);
            Vec center = center_of(state);
            R q[4];
            quat_of(state, q);
            Vec lin(R(state.linear[0]), R(state.linear[1]), R(state.linear[2]));
            Vec ang(R(state.angular[0]), R(state.angular[1]), R(state.angular[2]));
            known.center = center;
            known.velocity = lin;
            known.impulse = known.angular = Vec();
            for (const Vec& local : known.points) {
                Vec arm = rotate(q, local);
                m.start.push_back(center + arm);
                m.velocities.push_back(lin + cross(ang, arm));
                m.owners.push_back(uint32_t(owner));
            }
        }
        m.positions = m.start;
        movers = std::move(m);
        carry_movers(R(0));
    }

    // couple.rs:291-322: points `elapsed` into the step, sorted by (cell, owner, place) again
    void carry_movers(R elapsed) {
        size_t k = movers.start.size();
        struct MK {
            Key cell;
            uint32_t owner;
            size_t index;
        };
        std::vector<MK> order(k);
        for (size_t i = 0; i < k; ++i) {
            Vec at = movers.start[i] + movers.velocities[i] * elapsed;
            movers.positions[i] = at;
            order[i] = MK{cell_of(at), movers.owners[i], i};
        }
        std::sort(order.begin(), order.end(), [](const MK& a, const MK& b) {
            return std::tie(a.cell.x, a.cell.y, a.cell.z, a.owner, a.index) <
                   std::tie(b.cell.x, b.cell.y, b.cell.z, b.owner, b.index);
        });
        Movers m;
        std::vector<Key> keys(k);
        for (size_t i = 0; i < k; ++i) {
            size_t j = order[i].index;
            m.start.push_back(movers.start[j]);
            m.positions.push_back(movers.positions[j]);
            m.velocities.push_back(movers.velocities[j]);
            m.owners.push_back(movers.owners[j]);
            keys[i] = order[i].cell;
        }
        m.grid = Grid::build(keys);
        movers = std::move(m);
        for (auto& known : coupled) known.moved = known.velocity * elapsed;
    }

    // couple.rs:325-366: the fastest coupled body that may meet the water within dt
    R fastest_near_water(R dt, R slow) const {
        size_t count = coupled.size();
        std::vector<R> fastest_of(count, R(0));
        std::vector<Vec> lows(count, Vec::splat(R(FLT_MAX))), highs(count, Vec::splat(R(-FLT_MAX)));
        for (size_t i = 0; i < movers.positions.size(); ++i) {
            size_t owner = movers.owners[i];
            fastest_of[owner] = rmax(fastest_of[owner], length(movers.velocities[i]));
            lows[owner] = vmin(lows[owner], movers.positions[i]);
            highs[owner] = vmax(highs[owner], movers.positions[i]);
        }
        R water = fastest();
        R r = radius();
        R most = R(0);
        for (size_t b = 0; b < count; ++b) {
            R speed = fastest_of[b];
            if (speed <= most) continue;
            if (speed <= slow) {
                most = speed;
                continue;
            }
            Vec reach = Vec::splat(r + (speed + water) * dt);
            Key lo = cell_of(lows[b] - reach), hi = cell_of(highs[b] + reach);
            // before the first sort there is no grid to ask, any water counts
            bool wet = grid.cells.empty() && !positions.empty();
            for (size_t c = 0; !wet && c < grid.cells.size(); ++c) {
                const Key& k = grid.cells[c].first;
                wet = lo.x <= k.x && k.x <= hi.x && lo.y <= k.y && k.y <= hi.y && lo.z <= k.z && k.z <= hi.z;
            }
            if (wet) most = speed;
        }
        return most;
    }

    // couple.rs:375-416: pressure and damping between particle i and the body points near it;
    // adds what the particle feels to `push` and, given `bodies`, the damping's opposite to them
    void mover_push(size_t i, R mirrored, R damping, R settles, Vec& push, std::vector<std::pair<Vec, Vec>>* bodies) const {
        uint32_t b = mover_neighbors.start.empty() ? 0 : mover_neighbors.start[i];
        uint32_t e = mover_neighbors.start.empty() ? 0 : mover_neighbors.start[i + 1];
        if (b == e) return;
        Vec at = positions[i];
        Vec velocity = velocities[i];
        R density = densities[i];
        R r = radius();
        R soften = R(0.01f) * r * r;
        for (uint32_t k = b; k < e; ++k) {
            uint32_t point = mover_neighbors.items[k];
            Vec offset = at - movers.positions[point];
            Vec relative = velocity - movers.velocities[point];
            R toward = dot(relative, offset);
            R damp = toward < R(0) ? -damping * toward / (length_squared(offset) + soften) / density : R(0);
            Vec gradient = kernel.gradient(offset) * mass;
            push = push - gradient * (mirrored + damp);
            if (toward * toward < settles * length_squared(offset)) continue;
            if (!bodies) continue;
            Vec force = gradient * (damp * mass);
            uint32_t owner = movers.owners[point];
            const Coupled& known = coupled[owner];
            Vec arm = movers.positions[point] - (known.center + known.moved);
            (*bodies)[owner].first = (*bodies)[owner].first + force;
            (*bodies)[owner].second = (*bodies)[owner].second + cross(arm, force);
        }
    }

    // lift.rs:24-158: what the water does to each coupled body over dt, read as one smooth field
    struct Lift {
        size_t owner;
        Vec impulse, angular;
        std::vector<uint32_t> near;
    };
    std::vector<Lift> lifts(R dt, const Pose* poses, size_t npose) const {
        Vec g = gravity();
        R grav = length(g);
        Vec up = grav > R(0) ? (-g) / grav : Vec(R(0), R(1), R(0));
        R r = radius();
        R reach = R(3) * r;
        R column = r;
        std::vector<Lift> out;
        for (size_t owner = 0; owner < coupled.size(); ++owner) {
            const Coupled& known = coupled[owner];
            const Pose* state = pose_of(poses, npose, known.body);
            if (!state) continue;
            Vec center = center_of(*state);
            R q[4];
            quat_of(*state, q);
            Vec lin(R(state->linear[0]), R(state->linear[1]), R(state->linear[2]));
            Vec ang(R(state->angular[0]), R(state->angular[1]), R(state->angular[2]));
            std::vector<std::pair<Vec, Vec>> probes;
            for (const Vec& local : known.probes) {
                Vec arm = rotate(q, local);
                probes.push_back({arm, lin + cross(ang, arm)});
            }
            Vec low = Vec::splat(R(FLT_MAX)), high = Vec::splat(R(-FLT_MAX));
            for (auto& pr : probes) {
                low = vmin(low, center + pr.first);
                high = vmax(high, center + pr.first);
            }
            low = low - Vec::splat(reach);
            high = high + Vec::splat(reach);
            std::vector<uint32_t> near;
            for (size_t i = 0; i < len(); ++i)
                if (clamp(positions[i], low, high) == positions[i]) near.push_back(uint32_t(i));
            if (near.empty()) continue;
            // the level is the middle of the columns' tops
            struct Top {
                int32_t kx, kz;
                R h;
            };
            std::vector<Top> tops;
            for (uint32_t i : near) {
                Vec at = positions[i];
                tops.push_back(Top{as_i32(ofloor(at.x / column)), as_i32(ofloor(at.z / column)), dot(at, up)});
            }
            std::sort(tops.begin(), tops.end(), [](const Top& a, const Top& b) {
                if (a.kx != b.kx) return a.kx < b.kx;
                if (a.kz != b.kz) return a.kz < b.kz;
                return total_less(b.h, a.h);
            });
            std::vector<R> heights;
            for (size_t k = 0; k < tops.size(); ++k)
                if (k == 0 || tops[k].kx != tops[k - 1].kx || tops[k].kz != tops[k - 1].kz) heights.push_back(tops[k].h);
            std::sort(heights.begin(), heights.end(), [](R a, R b) { return total_less(a, b); });
            size_t quarter = heights.size() / 4;
            R sum = R(0);
            for (size_t k = quarter; k < heights.size() - quarter; ++k) sum += heights[k];
            R level = sum / R(float(heights.size() - 2 * quarter)) + R(settings.spacing) / R(2);
            Vec flow;
            uint32_t wet = 0;
            for (uint32_t i : near)
                if (dot(positions[i], up) <= level) {
                    flow = flow + velocities[i];
                    ++wet;
                }
            flow = flow / R(float(std::max<uint32_t>(wet, 1)));
            R spacing = known.probe_spacing;
            struct Under {
                Vec arm, velocity;
                R share;
            };
            std::vector<Under> under;
            for (auto& pr : probes) {
                R depth = level - dot(center + pr.first, up);
                R share = rmin(rmax(depth / spacing + R(0.5f), R(0)), R(1));
                if (share > R(0)) under.push_back(Under{pr.first, pr.second, share});
            }
            R wetted = R(0);
            for (auto& u : under) wetted += u.share;
            if (wetted <= R(0)) continue;
            R volume = wetted * (spacing * spacing * spacing);
            R density = R(settings.rest_density);
            Vec middle;
            for (auto& u : under) middle = middle + u.arm * u.share;
            middle = middle / wetted;
            Vec force, torque;
            Vec buoyancy = up * (density * grav * volume);
            force = force + buoyancy;
            torque = torque + cross(middle, buoyancy);
            R area = R(std::pow(volume, R(2.0f / 3.0f))) / wetted;
            for (auto& u : under) {
                Vec past = flow - u.velocity;
                Vec drag = past * (R(0.5f) * R(1) * density * area * u.share * length(past));
                force = force + drag;
                torque = torque + cross(u.arm, drag);
            }
            size_t nline = 0;
            for (auto& u : under) nline += u.share < R(1) ? 1 : 0;
            R plane = R(float(nline)) * spacing * spacing;
            R waves = density * plane * osqrt(grav * osqrt(plane));
            R share = waves / R(float(std::max<size_t>(nline, 1)));
            for (auto& u : under) {
                if (!(u.share < R(1))) continue;
                Vec calm = up * (share * dot(flow - u.velocity, up));
                force = force + calm;
                torque = torque + cross(u.arm, calm);
            }
            out.push_back(Lift{owner, force * dt, torque * dt, std::move(near)});
        }
        return out;
    }

    // lift.rs:160-166: the water read for a lift loses what the body got, shared by mass
    void give_back(const Lift& lift) {
        Vec change = lift.impulse / (mass * R(float(lift.near.size())));
        for (uint32_t i : lift.near) velocities[i] = velocities[i] - change;
    }

    // couple.rs:219-248 with the rigid world's part left to the caller: the bodies stand where
    // `poses` has them (a coupled body without a pose is uncoupled), and `pushes` receives, per
    // coupled body in body order, the lift (given back to the water when the body is dynamic)
    // and the damping impulse of the step, for the caller to apply as force and torque / dt
    Status step_with_bodies(R dt, const Pose* poses, size_t npose, Report& report, std::vector<Push>& pushes) {
        pushes.clear();
        if (settings.solver != 0 && !coupled.empty()) return INVALID_SETTINGS;
        place_movers_at(poses, npose);
        Status st = step(dt, report);
        movers = Movers{};
        // the points are gone: so are the lists into them
        if (!mover_neighbors.start.empty()) std::fill(mover_neighbors.start.begin(), mover_neighbors.start.end(), 0u);
        mover_neighbors.items.clear();
        if (st != OK) return st;
        for (auto& known : coupled) {
            Push p{};
            p.body = known.body;
            pushes.push_back(p);
        }
        if (dt > R(0)) {
            for (const Lift& lift : lifts(dt, poses, npose)) {
                Push& p = pushes[lift.owner];
                p.lift = lift.impulse;
                p.lift_angular = lift.angular;
                if (pose_of(poses, npose, coupled[lift.owner].body)->dynamic) {
                    give_back(lift);
                    p.lifted = 1;
                }
            }
            for (size_t b = 0; b < coupled.size(); ++b) {
                pushes[b].damping = coupled[b].impulse;
                pushes[b].damping_angular = coupled[b].angular;
                coupled[b].impulse = coupled[b].angular = Vec();
            }
        }
        return OK;
    }

    // flow.rs:109-113
    bool remove_flow(uint32_t id) {
        size_t before = flows.size();
        flows.erase(std::remove_if(flows.begin(), flows.end(), [&](const Flow& f) { return f.id == id; }),
                    flows.end());
        return flows.size() != before;
    }

    // mod.rs:468-486
    void keep_only(const std::vector<char>& keep) {
        size_t kept = 0;
        for (size_t i = 0; i < len(); ++i)
            if (keep[i]) {
                ids[kept] = ids[i];
                positions[kept] = positions[i];
                velocities[kept] = velocities[i];
                densities[kept] = densities[i];
                impulse[0][kept] = impulse[0][i];
                impulse[1][kept] = impulse[1][i];
                ++kept;
            }
        ids.resize(kept);
        positions.resize(kept);
        velocities.resize(kept);
        densities.resize(kept);
        impulse[0].resize(kept);
        impulse[1].resize(kept);
    }

    // Rust's `f as i64`: saturating, NaN to 0
    static int64_t as_i64(R v) {
        if (oisnan(v)) return 0;
        if (v >= R(9.2233720368547758e18)) return INT64_MAX;
        if (v <= R(-9.2233720368547758e18)) return INT64_MIN;
        return int64_t(v);
    }

    // Largest emitter lattice restated here: the reference allocates one flag per slot
    // (flow.rs:185) for up to 4096^3 slots; larger boxes are refused.
    static constexpr int64_t kMaxEmitterSlots = int64_t(1) << 30;

    // flow.rs:144-231: drains first, then emitters, each in the order they were added
    Status run_flows(uint32_t& emitted, uint32_t& drained) {
        emitted = drained = 0;
        if (flows.empty()) return OK;
        std::vector<Flow> list = flows;
        for (const Flow& flow : list) {
            if (flow.emitter) continue;
            std::vector<char> keep(len());
            size_t gone = 0;
            for (size_t i = 0; i < len(); ++i) {
                const Vec& at = positions[i];
                bool inside = at.x >= flow.low.x && at.y >= flow.low.y && at.z >= flow.low.z &&
                              at.x <= flow.high.x && at.y <= flow.high.y && at.z <= flow.high.z;
                keep[i] = !inside;
                gone += inside ? 1 : 0;
            }
            if (gone > 0) {
                drained += uint32_t(gone);
                keep_only(keep);
            }
        }
        const R spacing = R(settings.spacing);
        for (const Flow& flow : list) {
            if (!flow.emitter) continue;
            Vec size = flow.high - flow.low;
            auto count = [&](R extent) -> int64_t {
                int64_t c = as_i64(ofloor(extent / spacing));
                return std::min<int64_t>(std::max<int64_t>(c, 0), int64_t(1) << 12);
            };
            int64_t cx = count(size.x), cy = count(size.y), cz = count(size.z);
            int64_t total = cx * cy * cz;
            if (total == 0) continue;
            if (total > kMaxEmitterSlots) return OUT_OF_RANGE;
            R share = R(0.9f) * spacing;
            R clear = share * share;
            std::vector<char> taken(size_t(total), 0);
            for (const Vec& at : positions) {
                Vec local = (at - flow.low) / spacing - Vec::splat(R(0.5));
                // a slot index outside [-1, cells] reaches no slot; clamping keeps the loops finite
                auto nearest = [](R v, int64_t cells) {
                    int64_t c = as_i64(oround(v));
                    return std::min<int64_t>(std::max<int64_t>(c, -2), cells + 1);
                };
                int64_t nx = nearest(local.x, cx), ny = nearest(local.y, cy), nz = nearest(local.z, cz);
                for (int64_t y = ny - 1; y <= ny + 1; ++y)
                    for (int64_t z = nz - 1; z <= nz + 1; ++z)
                        for (int64_t x = nx - 1; x <= nx + 1; ++x) {
                            if (!(x >= 0 && x < cx && y >= 0 && y < cy && z >= 0 && z < cz)) continue;
                            Vec center = flow.low + Vec(R(x) + R(0.5), R(y) + R(0.5), R(z) + R(0.5)) * spacing;
                            if (length_squared(at - center) < clear) taken[size_t((y * cz + z) * cx + x)] = 1;
                        }
            }
            for (int64_t y = 0; y < cy; ++y)
                for (int64_t z = 0; z < cz; ++z)
                    for (int64_t x = 0; x < cx; ++x) {
                        if (taken[size_t((y * cz + z) * cx + x)]) continue;
                        Vec at = flow.low + Vec(R(x) + R(0.5), R(y) + R(0.5), R(z) + R(0.5)) * spacing;
                        Status st = add_particle(at, flow.velocity, nullptr);
                        if (st != OK) return st;
                        ++emitted;
                    }
        }
        return OK;
    }

    // mod.rs:493-524
    Status fill_box(Vec low, Vec high, uint64_t* count_out) {
        if (!is_finite(low) || !is_finite(high)) return NON_FINITE;
        if (high.x < low.x || high.y < low.y || high.z < low.z) return OUT_OF_RANGE;
        R spacing = R(settings.spacing);
        auto count = [&](R extent) -> uint64_t {
            R c = rmin(ofloor(extent / spacing), R(4294967295.0));
            if (oisnan(c) || c <= R(0)) return 0;
            return uint64_t(c);
        };
        Vec size = high - low;
        uint64_t nx = count(size.x), ny = count(size.y), nz = count(size.z);
        auto sat_mul = [](uint64_t a, uint64_t b) -> uint64_t {
            unsigned __int128 p = (unsigned __int128)a * b;
            return p > UINT64_MAX ? UINT64_MAX : uint64_t(p);
        };
        uint64_t total = sat_mul(sat_mul(nx, ny), nz);
        uint64_t room = settings.max_particles > len() ? settings.max_particles - len() : 0;
        uint64_t ids_left = uint64_t(UINT32_MAX - next_id);
        if (total > room || total > ids_left) return FLUID_FULL;
        Vec start = low + Vec::splat(spacing * R(0.5));
        for (uint64_t y = 0; y < ny; ++y)
            for (uint64_t z = 0; z < nz; ++z)
                for (uint64_t x = 0; x < nx; ++x) {
                    Vec at = start + Vec(R(x), R(y), R(z)) * spacing;
                    Status st = add_particle(at, Vec(), nullptr);
                    if (st != OK) return st;
                }
        if (count_out) *count_out = total;
        return OK;
    }

    // boundary.rs:230-238
    static Status check_box(Vec low, Vec high) {
        if (!is_finite(low) || !is_finite(high)) return NON_FINITE;
        if (high.x <= low.x || high.y <= low.y || high.z <= low.z) return OUT_OF_RANGE;
        return OK;
    }

    // boundary.rs:123-126 (f32::round rounds half away from zero)
    void cells_in(Vec extent, int64_t out[3]) const {
        auto count = [&](R length) -> int64_t {
            R c = rmin(oround(length / R(settings.spacing)), R(1e9));
            return int64_t(c);
        };
        out[0] = count(extent.x);
        out[1] = count(extent.y);
        out[2] = count(extent.z);
    }

    // boundary.rs:128-137
    Status check_room(int64_t count) const {
        uint64_t room = settings.max_particles > walls.positions.size()
                            ? settings.max_particles - walls.positions.size()
                            : 0;
        if (count < 0 || uint64_t(count) > room || walls.next == UINT32_MAX) return FLUID_FULL;
        return OK;
    }

    // boundary.rs:41-68
    Status add_box_container(Vec low, Vec high, uint32_t* id_out) {
        Status st = check_box(low, high);
        if (st != OK) return st;
        int64_t cells[3];
        cells_in(high - low, cells);
        int64_t layers = int64_t(oceil(settings.support));
        int64_t shell = (cells[0] + 2 * layers) * (cells[1] + 2 * layers) * (cells[2] + 2 * layers) -
                        cells[0] * cells[1] * cells[2];
        st = check_room(shell);
        if (st != OK) return st;
        R spacing = R(settings.spacing);
        std::vector<Vec> points;
        points.reserve(size_t(shell));
        for (int64_t y = -layers; y < cells[1] + layers; ++y)
            for (int64_t z = -layers; z < cells[2] + layers; ++z)
                for (int64_t x = -layers; x < cells[0] + layers; ++x) {
                    bool inside = x >= 0 && x < cells[0] && y >= 0 && y < cells[1] && z >= 0 && z < cells[2];
                    if (!inside) {
                        Vec at(R(float(x)) + R(0.5), R(float(y)) + R(0.5), R(float(z)) + R(0.5));
                        points.push_back(low + at * spacing);
                    }
                }
        uint32_t id = add_wall_points(points);
        walls.containers.push_back(Container<R>{id, low, high});
        update_bounds();
        if (id_out) *id_out = id;
        return OK;
    }

    // boundary.rs:74-91
    Status add_wall(Vec low, Vec high, uint32_t* id_out) {
        Status st = check_box(low, high);
        if (st != OK) return st;
        int64_t cells[3];
        cells_in(high - low, cells);
        for (auto& c : cells) c = std::max<int64_t>(c, 1);
        int64_t count = cells[0] * cells[1] * cells[2];
        st = check_room(count);
        if (st != OK) return st;
        R spacing = R(settings.spacing);
        std::vector<Vec> points;
        points.reserve(size_t(count));
        for (int64_t y = 0; y < cells[1]; ++y)
            for (int64_t z = 0; z < cells[2]; ++z)
                for (int64_t x = 0; x < cells[0]; ++x) {
                    Vec at(R(float(x)) + R(0.5), R(float(y)) + R(0.5), R(float(z)) + R(0.5));
                    points.push_back(low + at * spacing);
                }
        uint32_t id = add_wall_points(points);
        if (id_out) *id_out = id;
        return OK;
    }

    // boundary.rs:94-115
    bool remove_boundary(uint32_t id) {
        size_t before = walls.positions.size();
        size_t kept = 0;
        for (size_t i = 0; i < walls.positions.size(); ++i) {
            if (walls.owners[i] != id) {
                walls.positions[kept] = walls.positions[i];
                walls.owners[kept] = walls.owners[i];
                ++kept;
            }
        }
        walls.positions.resize(kept);
        walls.owners.resize(kept);
        bool had_container = false;
        std::vector<Container<R>> rest;
        for (auto& c : walls.containers) {
            if (c.id == id) had_container = true;
            else rest.push_back(c);
        }
        walls.containers = rest;
        update_bounds();
        size_t regions = terrains.size();
        terrains.erase(std::remove_if(terrains.begin(), terrains.end(), [&](const Terrain& t) { return t.owner == id; }),
                       terrains.end());
        bool gone = walls.positions.size() != before || had_container || terrains.size() != regions;
        if (gone) settle_walls();
        return gone;
    }

    // boundary.rs:240-247
    void update_bounds() {
        walls.has_bounds = false;
        for (auto& c : walls.containers) {
            if (!walls.has_bounds) {
                walls.bounds_low = c.low;
                walls.bounds_high = c.high;
                walls.has_bounds = true;
            } else {
                walls.bounds_low = vmin(walls.bounds_low, c.low);
                walls.bounds_high = vmax(walls.bounds_high, c.high);
            }
        }
    }

    uint32_t add_wall_points(const std::vector<Vec>& points) {
        uint32_t id = walls.next++;
        for (auto& p : points) {
            walls.positions.push_back(p);
            walls.owners.push_back(id);
        }
        settle_walls();
        return id;
    }

    Key cell_of(Vec p) const {
        Vec c = p / radius();
        return Key{sat_i32(ofloor(c.x)), sat_i32(ofloor(c.y)), sat_i32(ofloor(c.z))};
    }

    // boundary.rs:155-178: by cell, owner, position bits, then index.
    void settle_walls() {
        size_t n = walls.positions.size();
        struct WK {
            Key cell;
            uint32_t owner;
            uint64_t bx, by, bz;
            size_t index;
        };
        std::vector<WK> order(n);
        for (size_t i = 0; i < n; ++i) {
            Vec p = walls.positions[i];
            order[i] = WK{cell_of(p), walls.owners[i], bits_of(p.x), bits_of(p.y), bits_of(p.z), i};
        }
        std::sort(order.begin(), order.end(), [](const WK& a, const WK& b) {
            return std::tie(a.cell.x, a.cell.y, a.cell.z, a.owner, a.bx, a.by, a.bz, a.index) <
                   std::tie(b.cell.x, b.cell.y, b.cell.z, b.owner, b.bx, b.by, b.bz, b.index);
        });
        std::vector<Vec> pos(n);
        std::vector<uint32_t> own(n);
        std::vector<Key> keys(n);
        for (size_t i = 0; i < n; ++i) {
            pos[i] = walls.positions[order[i].index];
            own[i] = order[i].owner;
            keys[i] = order[i].cell;
        }
        walls.positions = std::move(pos);
        walls.owners = std::move(own);
        walls.grid = Grid::build(keys);
    }

    // mod.rs:264-277: indexes within `reach` of `at`, in range order.
    static void near(const std::vector<Vec>& pts, const std::vector<Range>& ranges, Vec at, R reach,
                     std::vector<uint32_t>& out) {
        for (const Range& r : ranges)
            for (uint32_t other = r.begin; other < r.end; ++other)
                if (length_squared(pts[other] - at) < reach) out.push_back(other);
    }

    // mod.rs:540-608
    void update_neighbors() {
        size_t n = len();
        struct OK_ {
            Key cell;
            uint32_t id, index;
        };
        std::vector<OK_> order(n);
        for (size_t i = 0; i < n; ++i) order[i] = OK_{cell_of(positions[i]), ids[i], uint32_t(i)};
        std::sort(order.begin(), order.end(), [](const OK_& a, const OK_& b) {
            return std::tie(a.cell.x, a.cell.y, a.cell.z, a.id, a.index) <
                   std::tie(b.cell.x, b.cell.y, b.cell.z, b.id, b.index);
        });
        std::vector<uint32_t> nid(n);
        std::vector<Vec> np(n), nv(n);
        std::vector<R> nd(n), nw0(n), nw1(n);
        std::vector<Key> keys(n);
        for (size_t i = 0; i < n; ++i) {
            uint32_t k = order[i].index;
            nid[i] = ids[k];
            np[i] = positions[k];
            nv[i] = velocities[k];
            nd[i] = densities[k];
            nw0[i] = impulse[0][k];
            nw1[i] = impulse[1][k];
            keys[i] = order[i].cell;
        }
        ids = std::move(nid);
        positions = std::move(np);
        velocities = std::move(nv);
        densities = std::move(nd);
        impulse[0] = std::move(nw0);
        impulse[1] = std::move(nw1);
        grid = Grid::build(keys);

        R reach = pow2(radius());
        std::vector<uint32_t> fcount(n), wcount(n), mcount(n);
        // lists are formed per particle; joining them in particle order is the chunked join of
        // mod.rs:294-307 without the chunk boundaries, which do not change the result
        std::vector<std::vector<uint32_t>> fparts, wparts, mparts;
        const size_t chunk = 512;
        size_t jobs = (n + chunk - 1) / chunk;
        fparts.resize(jobs);
        wparts.resize(jobs);
        mparts.resize(jobs);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads())
        for (long long job = 0; job < (long long)jobs; ++job) {
            std::vector<Range> af, aw, am;
            bool have = false;
            Key last{0, 0, 0};
            size_t b = size_t(job) * chunk, e = std::min(n, b + chunk);
            for (size_t i = b; i < e; ++i) {
                Vec at = positions[i];
                Key c = cell_of(at);
                if (!have || c != last) {
                    have = true;
                    last = c;
                    grid.around(c, af);
                    walls.grid.around(c, aw);
                    movers.grid.around(c, am);
                }
                size_t bf = fparts[job].size(), bw = wparts[job].size(), bm = mparts[job].size();
                near(positions, af, at, reach, fparts[job]);
                near(walls.positions, aw, at, reach, wparts[job]);
                near(movers.positions, am, at, reach, mparts[job]);
                fcount[i] = uint32_t(fparts[job].size() - bf);
                wcount[i] = uint32_t(wparts[job].size() - bw);
                mcount[i] = uint32_t(mparts[job].size() - bm);
            }
        }
        join(fcount, fparts, neighbors);
        join(wcount, wparts, wall_neighbors);
        join(mcount, mparts, mover_neighbors);
    }

    static void join(const std::vector<uint32_t>& counts, std::vector<std::vector<uint32_t>>& parts, Lists& out) {
        out.start.assign(counts.size() + 1, 0);
        for (size_t i = 0; i < counts.size(); ++i) out.start[i + 1] = out.start[i] + counts[i];
        out.items.clear();
        out.items.reserve(out.start.back());
        for (auto& p : parts) out.items.insert(out.items.end(), p.begin(), p.end());
    }

    int nthreads() const {
#ifdef _OPENMP
        return threads > 0 ? threads : omp_get_max_threads();
#else
        return 1;
#endif
    }

    // mod.rs:621-675
    Status compute_densities() {
        if (neighbors.start.size() != len() + 1) return OUT_OF_RANGE;
        size_t n = len();
        std::vector<R> out(n);
        std::vector<Vec> slopes(terrains.empty() ? 0 : n);
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            size_t i = size_t(ii);
            Vec at = positions[i];
            R sum = R(0);
            for (uint32_t k = neighbors.start[i]; k < neighbors.start[i + 1]; ++k)
                sum += kernel.value(length(positions[neighbors.items[k]] - at));
            R wsum = R(0);
            for (uint32_t k = wall_neighbors.start[i]; k < wall_neighbors.start[i + 1]; ++k)
                wsum += kernel.value(length(walls.positions[wall_neighbors.items[k]] - at));
            R msum = R(0);
            if (!mover_neighbors.start.empty())
                for (uint32_t k = mover_neighbors.start[i]; k < mover_neighbors.start[i + 1]; ++k)
                    msum += kernel.value(length(movers.positions[mover_neighbors.items[k]] - at));
            // ground_near (mod.rs:657-663): each region holding the particle adds its ground
            R ground = R(0);
            Vec slope;
            for (const Terrain& t : terrains) {
                R distance, density;
                Vec normal, gradient;
                if (!terrain_ground(t, at, distance, normal, density, gradient)) continue;
                ground = ground + density;
                slope = slope + gradient;
            }
            out[i] = mass * (sum + wsum + msum) + ground;
            if (!terrains.empty()) slopes[i] = slope;
        }
        densities = std::move(out);
        ground_slopes = terrains.empty() ? std::vector<Vec>() : std::move(slopes);
        return OK;
    }

    // mod.rs:677-691
    uint64_t state_hash() const {
        std::vector<size_t> order(len());
        std::iota(order.begin(), order.end(), size_t(0));
        std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return ids[a] < ids[b]; });
        std::vector<uint8_t> bytes;
        bytes.reserve(len() * 28);
        auto put32 = [&](uint32_t v) {
            for (int s = 0; s < 4; ++s) bytes.push_back(uint8_t(v >> (8 * s)));
        };
        for (size_t i : order) {
            put32(ids[i]);
            for (const Vec& v : {positions[i], velocities[i]}) {
                // the hash is of f32 bits; the double oracle hashes its values rounded to f32
                put32(uint32_t(bits_of(float(v.x))));
                put32(uint32_t(bits_of(float(v.y))));
                put32(uint32_t(bits_of(float(v.z))));
            }
        }
        return fnv1a(bytes.data(), bytes.size());
    }

    // ---- snapshots (save.rs) -------------------------------------------------------------------

    struct Out {
        std::vector<uint8_t> b;
        void u8(uint8_t v) { b.push_back(v); }
        void u32(uint32_t v) { for (int k = 0; k < 4; ++k) b.push_back(uint8_t((v >> (8 * k)) & 0xffu)); }
        void u64(uint64_t v) { for (int k = 0; k < 8; ++k) b.push_back(uint8_t((v >> (8 * k)) & 0xffu)); }
        void f32(float v) { u32(uint32_t(bits_of(v))); }
        void v3(const Vec& v) { f32(float(v.x)); f32(float(v.y)); f32(float(v.z)); }
    };

    // save.rs:18-73; vectors are stored as f32 (the double oracle rounds them)
    std::vector<uint8_t> save_snapshot() const {
        Out o;
        for (char c : {'S', 'L', 'F', 'L'}) o.u8(uint8_t(c));
        o.u32(3);
        o.u8(uint8_t(settings.solver));
        for (float v : {settings.spacing, settings.rest_density, settings.support, settings.sound_speed,
                        settings.viscosity, settings.courant})
            o.f32(v);
        o.u64(settings.max_particles);
        for (float g : settings.gravity) o.f32(g);
        o.u32(settings.max_substeps);
        o.u32(uint32_t(len()));
        for (size_t i = 0; i < len(); ++i) {
            o.u32(ids[i]);
            o.v3(positions[i]);
            o.v3(velocities[i]);
        }
        o.u32(next_id);
        o.u32(uint32_t(walls.positions.size()));
        for (size_t k = 0; k < walls.positions.size(); ++k) {
            o.v3(walls.positions[k]);
            o.u32(walls.owners[k]);
        }
        o.u32(walls.next);
        o.u32(uint32_t(walls.containers.size()));
        for (auto& c : walls.containers) {
            o.u32(c.id);
            o.v3(c.low);
            o.v3(c.high);
        }
        o.u32(uint32_t(flows.size()));
        for (auto& f : flows) {
            o.u32(f.id);
            o.v3(f.low);
            o.v3(f.high);
            o.u8(f.emitter ? 0 : 1);
            if (f.emitter) o.v3(f.velocity);
        }
        o.u32(flow_next);
        // Coupled::save (couple.rs:50-55)
        o.u32(uint32_t(coupled.size()));
        for (auto& c : coupled) {
            o.u32(uint32_t(c.body >> 32));
            o.u32(uint32_t(c.body & 0xffffffffu));
            o.u32(uint32_t(c.points.size()));
            for (auto& q : c.points) o.v3(q);
            o.f32(float(c.probe_spacing));
            o.u32(uint32_t(c.probes.size()));
            for (auto& q : c.probes) o.v3(q);
        }
        // TerrainField::save (terrain.rs:44-55)
        o.u32(uint32_t(terrains.size()));
        for (auto& t : terrains) {
            o.u32(t.owner);
            o.v3(t.low);
            o.u32(uint32_t(t.nx));
            o.u32(uint32_t(t.ny));
            o.u32(uint32_t(t.nz));
            o.f32(float(t.step));
            o.u32(uint32_t(t.distances.size()));
            for (R d : t.distances) o.f32(float(d));
        }
        o.u8(has_domain ? 1 : 0);
        if (has_domain) {
            o.v3(domain_low);
            o.v3(domain_high);
        }
        o.u64(fnv1a(o.b.data(), o.b.size()));
        return o.b;
    }

    struct In {
        const uint8_t* d;
        size_t n, at;
        std::string* msg;
        bool fail(const char* m) {
            if (msg->empty()) *msg = m;
            return false;
        }
        bool get(uint8_t* out, size_t k) {
            if (n - at < k) return fail("snapshot truncated");
            std::memcpy(out, d + at, k);
            at += k;
            return true;
        }
        bool u8(uint8_t& v) { return get(&v, 1); }
        bool u32(uint32_t& v) {
            uint8_t b[4];
            if (!get(b, 4)) return false;
            v = 0;
            for (int k = 3; k >= 0; --k) v = (v << 8) | b[k];
            return true;
        }
        bool u64(uint64_t& v) {
            uint8_t b[8];
            if (!get(b, 8)) return false;
            v = 0;
            for (int k = 7; k >= 0; --k) v = (v << 8) | b[k];
            return true;
        }
        bool f32(float& v) {
            uint32_t b;
            if (!u32(b)) return false;
            std::memcpy(&v, &b, 4);
            return true;
        }
        bool v3(Vec& v) {
            float x, y, z;
            if (!(f32(x) && f32(y) && f32(z))) return false;
            v = Vec(R(x), R(y), R(z));
            return true;
        }
        bool count(size_t record, uint64_t max, size_t& out) {
            uint32_t c;
            if (!u32(c)) return false;
            if (c > max) return fail("invalid snapshot: count over limit");
            if (uint64_t(c) * record > uint64_t(n - at)) return fail("snapshot truncated");
            out = c;
            return true;
        }
    };

    // save.rs:79-181 into `out`; `base` gives the fields the snapshot does not hold
    static Status load_snapshot(const uint8_t* data, size_t size, const Settings& base, World& out,
                                std::string& msg) {
        auto bad = [&](const std::string& m) {
            if (msg.empty()) msg = m;
            return SNAPSHOT;
        };
        if (size > (size_t(1) << 30)) return bad("snapshot over limit");
        if (size < 16) return bad("snapshot truncated");
        if (std::memcmp(data, "SLFL", 4) != 0) return bad("not a snapshot");
        size_t body = size - 8;
        uint64_t stored = 0;
        for (int k = 7; k >= 0; --k) stored = (stored << 8) | data[body + k];
        if (stored != fnv1a(data, body)) return bad("snapshot checksum mismatch");
        In r{data, body, 4, &msg};
        uint32_t version;
        if (!r.u32(version)) return SNAPSHOT;
        if (version < 1 || version > 3) return bad("unsupported snapshot version " + std::to_string(version));
        uint8_t solver;
        if (!r.u8(solver)) return SNAPSHOT;
        if (solver > 1) return bad("invalid snapshot: fluid solver");
        Settings st = base;
        st.solver = solver;
        float g[3];
        if (!(r.f32(st.spacing) && r.f32(st.rest_density) && r.f32(st.support) && r.f32(st.sound_speed) &&
              r.f32(st.viscosity) && r.f32(st.courant) && r.u64(st.max_particles) && r.f32(g[0]) && r.f32(g[1]) &&
              r.f32(g[2]) && r.u32(st.max_substeps)))
            return SNAPSHOT;
        for (int a = 0; a < 3; ++a) st.gravity[a] = g[a];
        World w;
        if (create(st, w) != OK) return bad("invalid snapshot: fluid settings");
        size_t count;
        if (!r.count(28, st.max_particles, count)) return SNAPSHOT;
        for (size_t i = 0; i < count; ++i) {
            uint32_t id;
            Vec at, v;
            if (!(r.u32(id) && r.v3(at) && r.v3(v))) return SNAPSHOT;
            if (!is_finite(at) || !is_finite(v)) return bad("invalid snapshot: fluid particle");
            w.ids.push_back(id);
            w.positions.push_back(at);
            w.velocities.push_back(v);
        }
        w.densities.assign(count, R(st.rest_density));
        w.impulse[0].assign(count, R(0));  // a loaded world starts cold
        w.impulse[1].assign(count, R(0));
        if (!r.u32(w.next_id)) return SNAPSHOT;
        std::vector<uint32_t> seen = w.ids;
        std::sort(seen.begin(), seen.end());
        for (size_t i = 1; i < seen.size(); ++i)
            if (seen[i] == seen[i - 1]) return bad("invalid snapshot: fluid particle id");
        if (!seen.empty() && seen.back() >= w.next_id) return bad("invalid snapshot: fluid particle id");
        size_t nw;
        if (!r.count(16, st.max_particles, nw)) return SNAPSHOT;
        for (size_t k = 0; k < nw; ++k) {
            Vec at;
            uint32_t owner;
            if (!r.v3(at)) return SNAPSHOT;
            if (!is_finite(at)) return bad("invalid snapshot: fluid wall");
            if (!r.u32(owner)) return SNAPSHOT;
            w.walls.positions.push_back(at);
            w.walls.owners.push_back(owner);
        }
        size_t nc;
        if (!(r.u32(w.walls.next) && r.count(28, st.max_particles, nc))) return SNAPSHOT;
        for (size_t k = 0; k < nc; ++k) {
            Container<R> c;
            if (!(r.u32(c.id) && r.v3(c.low) && r.v3(c.high))) return SNAPSHOT;
            if (check_box(c.low, c.high) != OK || c.id >= w.walls.next) return bad("invalid snapshot: fluid container");
            w.walls.containers.push_back(c);
        }
        for (uint32_t o : w.walls.owners)
            if (o >= w.walls.next) return bad("invalid snapshot: fluid wall owner");
        w.update_bounds();
        size_t nf;
        if (!r.count(29, 1 << 16, nf)) return SNAPSHOT;
        for (size_t k = 0; k < nf; ++k) {
            Flow f{};
            uint8_t kind;
            if (!(r.u32(f.id) && r.v3(f.low) && r.v3(f.high) && r.u8(kind))) return SNAPSHOT;
            if (kind == 0) {
                f.emitter = true;
                if (!r.v3(f.velocity)) return SNAPSHOT;
            } else if (kind != 1) {
                return bad("invalid snapshot: fluid flow kind");
            }
            bool inside_out = f.high.x <= f.low.x || f.high.y <= f.low.y || f.high.z <= f.low.z;
            if (!(is_finite(f.low) && is_finite(f.high) && is_finite(f.velocity)) || inside_out)
                return bad("invalid snapshot: fluid flow");
            w.flows.push_back(f);
        }
        if (!r.u32(w.flow_next)) return SNAPSHOT;
        for (auto& f : w.flows)
            if (f.id >= w.flow_next) return bad("invalid snapshot: fluid flow id");
        size_t ncoupled, terrains;
        if (!r.count(12, 1 << 16, ncoupled)) return SNAPSHOT;
        // Coupled::load (couple.rs:58-75), load_points (couple.rs:435-451)
        uint64_t room = st.max_particles;
        auto points = [&](uint64_t max, std::vector<Vec>& out) -> Status {
            size_t count;
            if (!r.count(12, max, count)) return SNAPSHOT;
            for (size_t k = 0; k < count; ++k) {
                Vec q;
                if (!r.v3(q)) return SNAPSHOT;
                if (!is_finite(q)) return bad("invalid snapshot: fluid body point");
                out.push_back(q);
            }
            if (out.empty()) return bad("invalid snapshot: fluid body");
            return OK;
        };
        for (size_t k = 0; k < ncoupled; ++k) {
            Coupled c;
            uint32_t index, generation;
            if (!(r.u32(index) && r.u32(generation))) return SNAPSHOT;
            c.body = (uint64_t(index) << 32) | generation;
            Status ps = points(room, c.points);
            if (ps != OK) return ps;
            if (version >= 3) {
                float ps2;
                if (!r.f32(ps2)) return SNAPSHOT;
                if (!oisfinite(ps2) || ps2 <= 0.0f) return bad("invalid snapshot: fluid body probes");
                c.probe_spacing = R(ps2);
                Status qs = points(kMaxProbes, c.probes);
                if (qs != OK) return qs;
            } else {
                c.probe_spacing = R(st.spacing);
                c.probes = c.points;
            }
            room -= c.points.size();
            w.coupled.push_back(std::move(c));
        }
        for (size_t k = 1; k < w.coupled.size(); ++k)
            if (w.coupled[k - 1].body >= w.coupled[k].body) return bad("invalid snapshot: fluid body order");
        if (!r.count(32, 1 << 16, terrains)) return SNAPSHOT;
        // TerrainField::load (terrain.rs:57-97)
        for (size_t k = 0; k < terrains; ++k) {
            Terrain t;
            uint32_t nx, ny, nz;
            float step;
            size_t count;
            if (!(r.u32(t.owner) && r.v3(t.low) && r.u32(nx) && r.u32(ny) && r.u32(nz) && r.f32(step) &&
                  r.count(4, kMaxTerrainNodes, count)))
                return SNAPSHOT;
            unsigned __int128 total = (unsigned __int128)nx * ny * nz;
            if (!is_finite(t.low) || !oisfinite(step) || step <= 0.0f || nx < 2 || ny < 2 || nz < 2 ||
                total != count)
                return bad("invalid snapshot: fluid terrain");
            t.nx = nx;
            t.ny = ny;
            t.nz = nz;
            t.step = R(step);
            for (size_t i = 0; i < count; ++i) {
                float d;
                if (!r.f32(d)) return SNAPSHOT;
                if (!oisfinite(d)) return bad("invalid snapshot: fluid terrain distance");
                t.distances.push_back(R(d));
            }
            if (t.owner >= w.walls.next) return bad("invalid snapshot: fluid terrain owner");
            w.terrains.push_back(std::move(t));
        }
        if (version >= 2) {
            uint8_t flag;
            if (!r.u8(flag)) return SNAPSHOT;
            if (flag > 1) return bad("invalid snapshot: fluid domain flag");
            if (flag == 1) {
                Vec lo, hi;
                if (!(r.v3(lo) && r.v3(hi))) return SNAPSHOT;
                if (w.set_domain(&lo, &hi) != OK) return bad("invalid snapshot: fluid domain");
            }
        }
        if (r.at != body) return bad("invalid snapshot: trailing bytes");
        w.settle_walls();
        out = std::move(w);
        return OK;
    }

    // step.rs:92-96
    R fastest() const {
        R most = R(0);
        for (auto& v : velocities) most = rmax(most, length(v));
        return most;
    }

    // step.rs:58-90
    Status step(R dt, Report& report) {
        report = Report();
        if (!oisfinite(dt) || dt < R(0)) return NON_FINITE;
        if (dt == R(0)) return OK;
        if (len() > 0) {
            Status st = settings.solver == 0 ? wcsph(dt, report) : dfsph(dt, report);
            if (st != OK) return st;
        }
        Status flowed = run_flows(report.emitted, report.drained);
        if (flowed != OK) return flowed;
        report.lost = keep_in_domain();
        report.max_speed = float(fastest());
        R rest = R(settings.rest_density);
        R most = R(0);
        for (auto d : densities) most = rmax(most, d / rest - R(1));
        report.max_compression = float(most);
        return OK;
    }

    // step.rs:102-116: the sound speed of the step follows the fastest coupled body near water
    Status wcsph(R dt, Report& report) {
        float configured = settings.sound_speed;
        R mover = fastest_near_water(dt, R(configured) / R(4));
        settings.sound_speed = float(rmax(R(configured), R(4) * mover));
        report.sound_speed = settings.sound_speed;
        Status st = wcsph_steps(dt, mover, report);
        settings.sound_speed = configured;
        return st;
    }

    // step.rs:118-142
    Status wcsph_steps(R dt, R mover, Report& report) {
        R fast = rmax(fastest(), mover);
        R largest = R(settings.courant) * radius() / (R(settings.sound_speed) + fast);
        R wanted = rmax(oceil(dt / largest), R(1));
        R cap = R(float(settings.max_substeps));
        uint32_t substeps = uint32_t(rmin(wanted, cap));
        report.capped = wanted > cap;
        R small = dt / R(float(substeps));
        for (uint32_t i = 0; i < substeps; ++i) {
            uint32_t held = 0;
            if (!coupled.empty()) carry_movers(small * R(float(i)));
            Status st = wcsph_substep(small, held);
            if (st != OK) return st;
            report.held_back += held;
        }
        report.substeps = substeps;
        return OK;
    }

    // step.rs:254-259
    R viscosity(R dt) const {
        R r = radius();
        return rmin(param(settings.viscosity, 0) * param(settings.sound_speed, 1) * r, R(0.05f) * r * r / dt);
    }

    // step.rs:262-301
    Vec wall_viscous(size_t index, R dt) const {
        R r = radius();
        R soften = R(0.01f) * r * r;
        R stable = r * r / dt;
        Vec at = positions[index];
        Vec velocity = velocities[index];
        R density = densities[index];
        Vec push;
        Vec away;
        for (uint32_t k = wall_neighbors.start[index]; k < wall_neighbors.start[index + 1]; ++k)
            away = away + (-kernel.gradient(at - walls.positions[wall_neighbors.items[k]]));
        Vec normal = normalize_or(away, Vec());
        Vec into = normal * rmin(dot(velocity, normal), R(0));
        R wall_visc = rmin(R(1) * param(settings.sound_speed, 1) * r, R(0.25f) * stable);
        for (const Terrain& t : terrains) {
            R distance;
            Vec n;
            if (!terrain_sample(t, at, distance, n)) continue;
            R towards = dot(velocity, n);
            if (towards < R(0)) {
                R weight = damping(distance);
                push = push - n * (wall_visc * towards * weight / density);
            }
        }
        for (uint32_t k = wall_neighbors.start[index]; k < wall_neighbors.start[index + 1]; ++k) {
            Vec offset = at - walls.positions[wall_neighbors.items[k]];
            R toward = dot(into, offset);
            if (toward < R(0)) {
                R squeeze = toward / (length_squared(offset) + soften);
                R damp = -wall_visc * squeeze / density;
                push = push - kernel.gradient(offset) * (mass * damp);
            }
        }
        return push;
    }

    // step.rs:229-251
    Vec viscous(size_t index, R dt) const {
        R r = radius();
        R soften = R(0.01f) * r * r;
        R visc = viscosity(dt);
        Vec at = positions[index];
        Vec velocity = velocities[index];
        R density = densities[index];
        Vec push;
        for (uint32_t k = neighbors.start[index]; k < neighbors.start[index + 1]; ++k) {
            uint32_t other = neighbors.items[k];
            if (other == index) continue;
            Vec offset = at - positions[other];
            R toward = dot(velocity - velocities[other], offset);
            if (toward < R(0)) {
                R squeeze = toward / (length_squared(offset) + soften);
                R damp = -visc * squeeze * R(2) / (density + densities[other]);
                push = push - kernel.gradient(offset) * (mass * damp);
            }
        }
        return constant_if(push, 64) + constant_if(wall_viscous(index, dt), 128);
    }

    // step.rs:144-224
    Status wcsph_substep(R dt, uint32_t& held) {
        update_neighbors();
        Status st = compute_densities();
        if (st != OK) return st;
        size_t n = len();
        R rest = R(settings.rest_density);
        R stiffness = rest * pow2(param(settings.sound_speed, 1)) / R(7);
        std::vector<R> pressures(n), scaled(n);
        for (size_t i = 0; i < n; ++i) {
            R ratio = rmin(densities[i] / rest, R(1.1f));
            pressures[i] = rmax(stiffness * (pow7(ratio) - R(1)), R(0));
        }
        for (size_t i = 0; i < n; ++i) scaled[i] = pressures[i] / (densities[i] * densities[i]);
        R r = radius();
        R soften = R(0.01f) * r * r;
        R visc = viscosity(dt);
        Vec g = gravity();
        // the body points' damping (step.rs:163-164) and the speed under which water settles
        // against them (couple.rs:390)
        R damping = rmin(R(1) * param(settings.sound_speed, 1) * r, R(0.25f) * r * r / dt);
        R settles = length(g) * R(settings.spacing);
        std::vector<Vec> pushes(n);
        std::vector<R> mirrors(coupled.empty() ? 0 : n);
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            size_t i = size_t(ii);
            Vec at = positions[i];
            Vec velocity = velocities[i];
            R density = densities[i];
            R own = scaled[i];
            Vec push;
            for (uint32_t k = neighbors.start[i]; k < neighbors.start[i + 1]; ++k) {
                uint32_t other = neighbors.items[k];
                Vec offset = at - positions[other];
                R squared = length_squared(offset);
                if (squared <= R(0)) continue;
                R distance = osqrt(squared);
                Vec gradient = offset * (kernel.slope(distance) / distance);
                R toward = rmin(dot(velocity - velocities[other], offset), R(0));
                R damp = -visc * toward / (squared + soften) * R(2) / (density + densities[other]);
                push = push - gradient * (mass * (own + scaled[other] + damp));
            }
            R mirrored = own + pressures[i] / (rest * rest);
            for (uint32_t k = wall_neighbors.start[i]; k < wall_neighbors.start[i + 1]; ++k) {
                Vec offset = at - walls.positions[wall_neighbors.items[k]];
                push = push - kernel.gradient(offset) * (mass * mirrored);
            }
            if (i < ground_slopes.size()) push = push - ground_slopes[i] * mirrored;
            mover_push(i, mirrored, damping, settles, push, nullptr);
            if (!mirrors.empty()) mirrors[i] = mirrored;
            pushes[i] = push + wall_viscous(i, dt) + g;
        }
        // what the body points took: summed per 512-particle chunk in particle order, the
        // chunks' sums added in order (step.rs:173-221)
        if (!coupled.empty()) {
            for (size_t c0 = 0; c0 < n; c0 += 512) {
                std::vector<std::pair<Vec, Vec>> felt(coupled.size());
                Vec unused;
                for (size_t i = c0; i < std::min(n, c0 + 512); ++i)
                    mover_push(i, mirrors[i], damping, settles, unused, &felt);
                for (size_t b = 0; b < coupled.size(); ++b) {
                    coupled[b].impulse = coupled[b].impulse + felt[b].first * dt;
                    coupled[b].angular = coupled[b].angular + felt[b].second * dt;
                }
            }
        }
        for (size_t i = 0; i < n; ++i) velocities[i] = velocities[i] + pushes[i] * dt;
        return advance(dt, held);
    }

    // step.rs:305-339.  A non-finite particle stops the pass there, as in the reference; earlier
    // particles have moved.
    Status advance(R dt, uint32_t& held) {
        held = 0;
        Vec rest = Vec::splat(R(settings.spacing) / R(2));
        for (size_t i = 0; i < len(); ++i) {
            Vec& at = positions[i];
            Vec& velocity = velocities[i];
            Vec next = at + velocity * dt;
            if (walls.has_bounds) {
                Vec low = walls.bounds_low, high = walls.bounds_high;
                Vec inside = clamp(next, low + rest, high - rest);
                if (inside != next) {
                    if (clamp(next, low, high) != next) held += 1;
                    if (inside.x != next.x) velocity.x = R(0);
                    if (inside.y != next.y) velocity.y = R(0);
                    if (inside.z != next.z) velocity.z = R(0);
                    next = inside;
                }
            }
            if (terrain_contact(rest.x, next, velocity)) held += 1;
            if (!is_finite(next) || !is_finite(velocity)) return NON_FINITE;
            at = next;
        }
        return OK;
    }

    // ---- DFSPH (dfsph.rs) ----------------------------------------------------------------

    // dfsph.rs:46-77
    Status dfsph(R dt, Report& report) {
        // dfsph.rs:52-55: ground pushes through the weakly compressible solver's pressure only
        if (!terrains.empty()) return INVALID_SETTINGS;
        R spacing = R(settings.spacing);
        R courant = R(settings.courant);
        R pull = length(gravity());
        R left = dt;
        while (left > R(0)) {
            R small = courant * spacing / rmax(fastest(), R(1e-6f));
            if (pull > R(0)) small = rmin(small, osqrt(R(2) * courant * spacing / pull));
            if (report.substeps + 1 >= settings.max_substeps && small < left) {
                report.capped = 1;
                small = left;
            }
            small = rmin(small, left);
            uint32_t held = 0, iterations = 0;
            Status st = dfsph_substep(small, held, iterations);
            if (st != OK) return st;
            report.iterations += iterations;
            report.held_back += held;
            report.substeps += 1;
            left -= small;
        }
        return OK;
    }

    // dfsph.rs:108-136
    void gradients() {
        grad_fluid.resize(neighbors.items.size());
        grad_walls.resize(wall_neighbors.items.size());
        size_t n = len();
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            size_t i = size_t(ii);
            Vec at = positions[i];
            for (uint32_t k = neighbors.start[i]; k < neighbors.start[i + 1]; ++k)
                grad_fluid[k] = constant_if(kernel.gradient(at - positions[neighbors.items[k]]), 1);
            for (uint32_t k = wall_neighbors.start[i]; k < wall_neighbors.start[i + 1]; ++k)
                grad_walls[k] = constant_if(kernel.gradient(at - walls.positions[wall_neighbors.items[k]]), 2);
        }
    }

    // dfsph.rs:138-163
    std::vector<R> factors() const {
        size_t n = len();
        std::vector<R> out(n);
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            size_t i = size_t(ii);
            Vec sum;
            R squares = R(0);
            for (uint32_t k = neighbors.start[i]; k < neighbors.start[i + 1]; ++k) {
                Vec part = grad_fluid[k] * mass;
                sum = sum + part;
                squares += length_squared(part);
            }
            for (uint32_t k = wall_neighbors.start[i]; k < wall_neighbors.start[i + 1]; ++k)
                sum = sum + grad_walls[k] * mass;
            R total = length_squared(sum) + squares;
            out[i] = constant_if(total > R(0) ? R(1) / total : R(0), 4);
        }
        return out;
    }

    // dfsph.rs:166-181
    R density_rate(size_t i) const {
        Vec velocity = velocities[i];
        R rate = R(0);
        for (uint32_t k = neighbors.start[i]; k < neighbors.start[i + 1]; ++k)
            rate += dot(velocity - velocities[neighbors.items[k]], grad_fluid[k]);
        for (uint32_t k = wall_neighbors.start[i]; k < wall_neighbors.start[i + 1]; ++k)
            rate += dot(velocity, grad_walls[k]);
        return rate * mass;
    }

    // dfsph.rs:184-216
    void push_apart(const std::vector<R>& stiffness, R dt) {
        size_t n = len();
        std::vector<Vec> changes(n);
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) {
            size_t i = size_t(ii);
            R own = stiffness[i];
            Vec change;
            for (uint32_t k = neighbors.start[i]; k < neighbors.start[i + 1]; ++k)
                change = change - grad_fluid[k] * (mass * (own + stiffness[neighbors.items[k]]));
            for (uint32_t k = wall_neighbors.start[i]; k < wall_neighbors.start[i + 1]; ++k)
                change = change - grad_walls[k] * (mass * own);
            changes[i] = change * dt;
        }
        for (size_t i = 0; i < n; ++i) velocities[i] = velocities[i] + changes[i];
    }

    // dfsph.rs:222-275; solve 0 = divergence, 1 = density
    uint32_t solve(int which, R dt, const std::vector<R>& alpha) {
        R rest = R(settings.rest_density);
        size_t n = len();
        R tolerance = which == 0 ? R(settings.divergence_tolerance) : R(settings.density_tolerance);
        uint32_t iterations = 0;
        std::vector<R> stiffness(n), errors(n);
        std::vector<R>& applied = impulse[which];
        if (settings.warm_start) {
            // the stiffness that applies half the last solve's impulse at this dt, pushed once;
            // the impulse restarts from it
            for (size_t i = 0; i < n; ++i) {
                stiffness[i] = (R(0.5f) * applied[i]) / dt;
                applied[i] = stiffness[i] * dt;
            }
            push_apart(stiffness, dt);
        }
        for (;;) {
#pragma omp parallel for schedule(static) num_threads(nthreads())
            for (long long ii = 0; ii < (long long)n; ++ii) {
                size_t i = size_t(ii);
                R rate = density_rate(i);
                R target, error;
                if (which == 1) {
                    R over = rmax(densities[i] + dt * rate - rest, R(0));
                    target = over / (dt * dt);
                    error = over / rest;
                } else {
                    size_t crowd = neighbors.count(i) + wall_neighbors.count(i);
                    R r = crowd < 20 ? R(0) : rmax(rate, R(0));
                    target = r / dt;
                    error = dt * r / rest;
                }
                stiffness[i] = constant_if(target * alpha[i], 32);
                errors[i] = error;
            }
            size_t loaded = 0;
            for (auto e : errors) loaded += e > R(0) ? 1 : 0;
            if (loaded == 0) loaded = 1;
            bool settled;
            if (settings.residual_sum == 0) {
                R sum = R(0);
                for (auto e : errors) sum += e;
                R average = sum / R(float(loaded));
                settled = iterations >= settings.min_iterations && average <= tolerance;
            } else {
                CompensatedSum acc;
                for (auto e : errors) acc.add(double(e));
                double average = acc.value() / double(loaded);
                settled = iterations >= settings.min_iterations && average <= double(tolerance);
            }
            // a derivative run held to another run's solves stops where that run stopped
            if (forced_next < forced_iterations.size()) settled = iterations >= forced_iterations[forced_next];
            if (settled || iterations >= settings.max_iterations) {
                if (forced_next < forced_iterations.size()) ++forced_next;
                return iterations;
            }
            push_apart(stiffness, dt);
            if (settings.warm_start)
                for (size_t i = 0; i < n; ++i) applied[i] = applied[i] + stiffness[i] * dt;
            iterations += 1;
        }
    }

    // dfsph.rs:79-103
    Status dfsph_substep(R dt, uint32_t& held, uint32_t& iterations) {
        update_neighbors();
        Status st = compute_densities();
        if (st != OK) return st;
        if (hold & 8)
            for (auto& d : densities) d = constant_if(d, 8);
        gradients();
        std::vector<R> alpha = factors();
        last_iterations[0] = solve(0, dt, alpha);
        iterations = last_iterations[0];
        size_t n = len();
        Vec g = gravity();
        std::vector<Vec> pushes(n);
#pragma omp parallel for schedule(static) num_threads(nthreads())
        for (long long ii = 0; ii < (long long)n; ++ii) pushes[size_t(ii)] = constant_if(viscous(size_t(ii), dt) + g, 16);
        for (size_t i = 0; i < n; ++i) velocities[i] = velocities[i] + pushes[i] * dt;
        last_iterations[1] = solve(1, dt, alpha);
        iterations += last_iterations[1];
        return advance(dt, held);
    }
};

}  // namespace oracle
