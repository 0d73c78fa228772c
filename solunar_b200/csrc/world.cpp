// world.cpp -- the host side of the library: FluidWorld's state owner and the C ABI.
//
// The world holds settings and walls on the host (walls are static and built once, as the
// reference builds them, src/fluid/boundary.rs) and every particle array on the device.  A step
// launches the substep kernels on the world's stream and reads back one small status block per
// substep, which carries what the host decides on: the bounding box of cells for the next sort,
// the fastest particle (substep length), the solver's stop flag, non-finite and held-back counts.
//
// Buffer discipline: the committed particle state is never written by a substep.  The sort
// copies it into a second slot, the substep works there and in a third, and only a substep that
// finished clean is committed by switching slot indexes.  A failed substep therefore leaves the
// particles as the last finished substep put them (src/fluid/step.rs:55-57).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/solunar_fluid.h"

// EXACT DFSPH keeps each pair's gradient for the solver check (0: the check gathers positions)
#ifndef SLF_KEEP_GRADIENTS
#define SLF_KEEP_GRADIENTS 1
#endif
#include "launch.h"

namespace slf {
namespace {

thread_local std::string g_error;

int32_t fail(int32_t code, const std::string& msg) {
    g_error = msg;
    return code;
}

#define SLF_CUDA(expr)                                                                            \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess) return fail(SLF_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define SLF_TRY(expr)                 \
    do {                              \
        int32_t st_ = (expr);         \
        if (st_ != SLF_OK) return st_; \
    } while (0)

// Device array that grows geometrically.
template <class T> struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;
    int32_t ensure(size_t n, size_t keep, cudaStream_t s) {
        if (n <= cap) return SLF_OK;
        size_t want = std::max<size_t>(n, cap + cap / 2);
        want = std::max<size_t>(want, 256);
        T* q = nullptr;
        SLF_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&q), want * sizeof(T), s));
        if (p && keep) SLF_CUDA(cudaMemcpyAsync(q, p, std::min(keep, cap) * sizeof(T), cudaMemcpyDeviceToDevice, s));
        if (p) SLF_CUDA(cudaFreeAsync(p, s));
        p = q;
        cap = want;
        return SLF_OK;
    }
    void release(cudaStream_t s) {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        cap = 0;
    }
};

// ---- host arithmetic in the reference's f32 order ------------------------------------------

inline float pow3f(float x) { return x * (x * x); }
inline float pow4f(float x) { float s = x * x; return s * s; }

struct HostKernel {
    float radius, scale;
    explicit HostKernel(float r) : radius(r), scale(21.0f / (2.0f * 3.14159265358979323846f * pow3f(r))) {}
    float value(float d) const {
        float q = d / radius;
        if (q >= 1.0f) return 0.0f;
        return scale * pow4f(1.0f - q) * (1.0f + 4.0f * q);
    }
    // Kernel::slope (mod.rs:149-155)
    float slope(float d) const {
        float q = d / radius;
        if (q >= 1.0f) return 0.0f;
        return scale * -20.0f * q * pow3f(1.0f - q) / radius;
    }
};

inline float rmin(float a, float b) {
    if (std::isnan(a)) return b;
    if (std::isnan(b)) return a;
    return b < a ? b : a;
}
inline float rmax(float a, float b) {
    if (std::isnan(a)) return b;
    if (std::isnan(b)) return a;
    return b > a ? b : a;
}

inline int32_t sat_i32(float v) {
    if (std::isnan(v)) return 0;
    if (v >= 2147483647.0f) return INT32_MAX;
    if (v <= -2147483648.0f) return INT32_MIN;
    return static_cast<int32_t>(v);
}

struct F3 {
    float x, y, z;
};
// f32 vector arithmetic of the coupled bodies' host-side steps, in the reference's order
inline F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3 operator-(F3 a) { return {-a.x, -a.y, -a.z}; }
inline F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline F3 operator/(F3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline bool operator==(F3 a, F3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(F3 a) { return std::sqrt(dot(a, a)); }
inline F3 vmin(F3 a, F3 b) { return {rmin(a.x, b.x), rmin(a.y, b.y), rmin(a.z, b.z)}; }
inline F3 vmax(F3 a, F3 b) { return {rmax(a.x, b.x), rmax(a.y, b.y), rmax(a.z, b.z)}; }
// f32::total_cmp's order
inline bool total_less(float a, float b) {
    int32_t x, y;
    std::memcpy(&x, &a, 4);
    std::memcpy(&y, &b, 4);
    x ^= int32_t(uint32_t(x >> 31) >> 1);
    y ^= int32_t(uint32_t(y >> 31) >> 1);
    return x < y;
}
inline F3 cross(F3 a, F3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
// q * v for the unit quaternion (x, y, z, w): v (w^2 - |b|^2) + b 2 (v.b) + (b x v) 2 w, b = (x, y, z)
inline F3 rotate(const float q[4], F3 v) {
    F3 b{q[0], q[1], q[2]};
    float w = q[3];
    float b2 = dot(b, b);
    return v * (w * w - b2) + b * (dot(v, b) * 2.0f) + cross(b, v) * (w * 2.0f);
}
inline bool finite3(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

struct Key3 {
    int32_t x, y, z;
    bool operator==(const Key3& o) const { return x == o.x && y == o.y && z == o.z; }
    bool operator<(const Key3& o) const { return std::tie(x, y, z) < std::tie(o.x, o.y, o.z); }
};

struct ContainerBox {
    uint32_t id;
    F3 low, high;
};

// Per-kernel device time from CUDA events bracketing each launch (while enabled).
struct Profiler {
    bool on = false;
    std::vector<std::string> names;
    std::vector<uint64_t> launches;
    std::vector<double> ms, bytes;
    struct Pending {
        int kind;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;

    int kind(const char* name) {
        for (size_t i = 0; i < names.size(); ++i)
            if (names[i] == name) return int(i);
        names.emplace_back(name);
        launches.push_back(0);
        ms.push_back(0.0);
        bytes.push_back(0.0);
        return int(names.size() - 1);
    }
    cudaEvent_t take() {
        if (pool.empty()) {
            cudaEvent_t e = nullptr;
            cudaEventCreate(&e);
            return e;
        }
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    // after a synchronisation of the stream: every pending pair has completed
    void collect() {
        for (auto& p : pending) {
            float t = 0.0f;
            if (cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) {
                ms[p.kind] += t;
                launches[p.kind] += 1;
                bytes[p.kind] += p.bytes;
            }
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    void reset() {
        for (size_t i = 0; i < names.size(); ++i) {
            launches[i] = 0;
            ms[i] = 0.0;
            bytes[i] = 0.0;
        }
    }
    ~Profiler() {
        for (auto& p : pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

// Algorithmic bytes a particle costs in each kernel: one read or write of every particle field
// the pass must touch, neighbour gathers served on chip not counted (f32 fields, 12-byte
// vectors).  The spatial hash's 72 bytes (read position, velocity, id; write them sorted; write
// and read the cell key) are split over its kernels.
namespace bytes_per_particle {
constexpr double count_cells = 20, scan = 2, scatter = 8, reorder = 44;
constexpr double density_wcsph = 16, density_dfsph = 20, wcsph_force = 52;
constexpr double rate_divergence = 32, rate_density = 36, push = 40, viscosity = 40, advance = 48;
constexpr double stats = 24;
constexpr double walk_order = 4;  // one row index written a particle
}  // namespace bytes_per_particle

}  // namespace

// ---- snapshot bytes (src/snapshot/bytes.rs): little-endian, f32 as its bits, lengths as u32 ----

inline uint64_t fnv1a64(const uint8_t* data, size_t n) {
    uint64_t h = 0xcbf29ce484222325ull;
    for (size_t i = 0; i < n; ++i) {
        h ^= uint64_t(data[i]);
        h *= 0x00000100000001b3ull;
    }
    return h;
}

struct SnapWriter {
    std::vector<uint8_t> data;
    void bytes(const void* p, size_t n) {
        const uint8_t* b = static_cast<const uint8_t*>(p);
        data.insert(data.end(), b, b + n);
    }
    void u8(uint8_t v) { data.push_back(v); }
    void u32(uint32_t v) {
        for (int k = 0; k < 4; ++k) data.push_back(uint8_t(v >> (8 * k)));
    }
    void u64(uint64_t v) {
        for (int k = 0; k < 8; ++k) data.push_back(uint8_t(v >> (8 * k)));
    }
    void f32(float v) {
        uint32_t b;
        std::memcpy(&b, &v, 4);
        u32(b);
    }
    void len(size_t v) { u32(uint32_t(v)); }
    void vec3(float x, float y, float z) {
        f32(x);
        f32(y);
        f32(z);
    }
};

// Reads untrusted bytes: every read checks what is left; a failure sets `error` to the
// reference's message (SnapshotError's Display, src/snapshot/mod.rs:65-76) and returns false.
struct SnapReader {
    const uint8_t* data;
    size_t size, at;
    std::string error;
    bool take(void* out, size_t n) {
        if (n > size - at) return fail_with("snapshot truncated");
        std::memcpy(out, data + at, n);
        at += n;
        return true;
    }
    bool fail_with(const char* m) {
        if (error.empty()) error = m;
        return false;
    }
    bool u8(uint8_t& v) { return take(&v, 1); }
    bool u32(uint32_t& v) {
        uint8_t b[4];
        if (!take(b, 4)) return false;
        v = uint32_t(b[0]) | uint32_t(b[1]) << 8 | uint32_t(b[2]) << 16 | uint32_t(b[3]) << 24;
        return true;
    }
    bool u64(uint64_t& v) {
        uint32_t lo, hi;
        if (!u32(lo) || !u32(hi)) return false;
        v = uint64_t(lo) | uint64_t(hi) << 32;
        return true;
    }
    bool f32(float& v) {
        uint32_t b;
        if (!u32(b)) return false;
        std::memcpy(&v, &b, 4);
        return true;
    }
    bool vec3(F3& v) { return f32(v.x) && f32(v.y) && f32(v.z); }
    // Reader::count (bytes.rs:133-150): the count against `max` and the bytes left
    bool count(size_t record, size_t max, size_t& out) {
        uint32_t c;
        if (!u32(c)) return false;
        if (c > max) return fail_with("invalid snapshot: count over limit");
        if ((unsigned __int128)c * record > (unsigned __int128)(size - at)) return fail_with("snapshot truncated");
        out = c;
        return true;
    }
};

inline bool finite3f(const F3& v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }

constexpr uint32_t kSnapshotVersion = 3;           // FLUID_SNAPSHOT_VERSION (save.rs:9)
constexpr size_t kMaxSnapshotBytes = size_t(1) << 30;  // MAX_FLUID_SNAPSHOT_BYTES (save.rs:12)
constexpr size_t kMaxSnapshotParts = size_t(1) << 16;  // MAX_PARTS (save.rs:14)

struct World {
    slf_settings s{};
    float radius = 0, mass = 0, scale = 0;
    cudaStream_t stream = nullptr;

    // particles
    uint64_t n = 0;
    uint32_t next_id = 0;
    std::vector<float4> pend_pos, pend_vel;
    std::vector<uint32_t> pend_ids;
    int cpos = 0, cid = 0;  // committed slots of pos/vel (of 3) and ids/rho (of 2)
    DevBuf<float4> pos[3], vel[3];
    DevBuf<int4> cell[3];  // cell-relative positions: the cell of each pos slot's offsets
    DevBuf<uint32_t> ids[2];
    DevBuf<float> rho[2];
    // warm starts: per particle the stiffness impulse (sum of kappa dt) its last divergence (x)
    // and density (y) solve applied; slotted with ids/rho, carried through sorts and compactions
    DevBuf<float2> warm[2];
    DevBuf<float> press, scaled, alpha;
    DevBuf<uint32_t> lin, cslot, members, count, tiles, keep;
    // neighbour lists of the current substep (fluid and walls)
    DevBuf<uint2> fent, went;
    // EXACT DFSPH: each pair's kernel gradient at the same slots (PairLists::gv), for the check
    DevBuf<float4> fgv, wgv;
    DevBuf<uint32_t> fcnt, wcnt;
    uint32_t list_cap = 0;
    DevBuf<uint8_t> partials;
    bool stats_fresh = false;  // status holds bbox and speed of the committed state

    // fluid cell table of the last sort, and the list passes' walk order over it
    GridDev fgrid{};
    DevBuf<uint32_t> worder, wkeys, wsums;
    bool worder_valid = false;
    int lists_pos = -1;  // slot of the positions the last sort produced
    uint64_t lists_n = 0;
    bool lists_valid = false;

    // walls
    std::vector<F3> wpos;
    std::vector<uint32_t> wown;
    uint32_t wall_next = 0;
    std::vector<ContainerBox> containers;
    bool has_bounds = false;
    F3 blow{}, bhigh{};
    DevBuf<float4> dwalls;
    DevBuf<uint32_t> dwstart;
    DevBuf<int4> dwkeys;
    GridDev wgrid{};
    bool walls_dirty = true;

    bool has_domain = false;
    F3 dlow{}, dhigh{};

    // terrain regions (terrain.rs:36-42) and the ground sites (terrain.rs:176-186)
    struct TerrainHost {
        uint32_t owner;
        F3 low;
        uint32_t nx, ny, nz;
        float step;
        std::vector<float> distances;
    };
    std::vector<TerrainHost> terrains;
    std::vector<float4> site_host;
    std::vector<float> far_host, damping_host;
    float ground_reach = 0, ground_low = 0, ground_step = 0;
    DevBuf<TerrainRegion> dregions;
    DevBuf<float> ddist, dfar, ddamping;
    DevBuf<float4> dsites, gslope;
    bool terrain_dirty = true;
    TerrainDev tdev{};

    Status* d_status = nullptr;
    Status* h_status = nullptr;
    Status* h_reset = nullptr;  // pinned: the status a substep starts from (a graph copies it)
    StepConsts* d_consts = nullptr;

    int64_t skip_job = -1;  // testing: next sort leaves this 512-particle job undone
    // set while the adjoint recomputes a substep: the sort's destinations, the pre-clamp velocity
    uint32_t* sort_dest = nullptr;
    float4* vel_pre = nullptr;

    // What the adjoint of a DFSPH substep needs beyond the substep's sort and densities: each
    // solver iteration's density rates and the velocities its check read, the velocities the
    // viscosity read and the advance's clamp flags.
    struct DfsphRecord {
        DevBuf<float4> div_vel, den_vel, va, pre;
        DevBuf<float> div_rate, den_rate;
        uint32_t div_n = 0, den_n = 0;
        void release(cudaStream_t st) {
            for (auto* b : {&div_vel, &den_vel, &va, &pre}) b->release(st);
            div_rate.release(st);
            den_rate.release(st);
        }
    };
    // A substep recorded as it ran (tapes that checkpoint every substep's record): the state
    // before it and its solver record.
    struct SubRecord {
        float dt = 0.0f;
        DevBuf<float4> pos, vel;
        DevBuf<uint32_t> ids;
        DfsphRecord rec;
        void release(cudaStream_t st) {
            pos.release(st);
            vel.release(st);
            ids.release(st);
            rec.release(st);
        }
    };

    // ---- the tape of slf_tape_begin: checkpoints and the substep lengths of each step ----
    struct Tape {
        bool on = false;
        uint32_t every = 1;
        uint64_t n = 0;
        std::vector<std::vector<float>> steps;  // substep lengths of each recorded step
        std::vector<size_t> ckpt_step;          // checkpoint c = the state before step ckpt_step[c]
        DevBuf<float4> cpos, cvel;              // [c][n]
        DevBuf<uint32_t> cids;
        std::vector<std::unique_ptr<SubRecord>> subs;  // every == 0: each substep's record
    } tape;
    // Records of finished tapes and segments, kept with their device buffers for the next ones:
    // the rounds of an optimisation loop then record without allocating (tens of GB at a
    // million particles, whose first allocation costs far more than the steps).
    std::vector<std::unique_ptr<SubRecord>> spare_records;
    // scratch of slf_step_backward
    struct BackScratch {
        DevBuf<float4> spos, svel, xo, vo, xp, vp, ab, xb, vb, pre, gt, kw, vr;
        DevBuf<uint32_t> sids, dest;
        DevBuf<float> srho, rb, abar, zeros;
        DevBuf<double> grads;
        void release(cudaStream_t s) {
            for (auto* b : {&spos, &svel, &xo, &vo, &xp, &vp, &ab, &xb, &vb, &pre, &gt, &kw, &vr}) b->release(s);
            for (auto* b : {&srho, &rb, &abar, &zeros}) b->release(s);
            sids.release(s);
            dest.release(s);
            grads.release(s);
        }
    } back;
    std::unique_ptr<SubRecord> new_record() {
        if (spare_records.empty()) return std::make_unique<SubRecord>();
        auto r = std::move(spare_records.back());
        spare_records.pop_back();
        return r;
    }
    std::vector<float>* tape_step = nullptr;  // the step being recorded
    Profiler prof;
    DevBuf<float> stage;  // xyz triples for host copies

    template <class F> void timed(const char* name, double per_particle, F&& f) {
        if (!prof.on) {
            f();
            return;
        }
        Profiler::Pending pd{prof.kind(name), prof.take(), prof.take(), per_particle * double(n)};
        cudaEventRecord(pd.a, stream);
        f();
        cudaEventRecord(pd.b, stream);
        prof.pending.push_back(pd);
    }

    int32_t sync() {
        SLF_CUDA(cudaStreamSynchronize(stream));
        prof.collect();
        return SLF_OK;
    }

    ~World() {
        if (stream) {
            for (auto* b : {&pos[0], &pos[1], &pos[2], &vel[0], &vel[1], &vel[2]}) b->release(stream);
            for (auto* b : {&ids[0], &ids[1], &lin, &cslot, &members, &count, &tiles, &keep, &dwstart, &fcnt, &wcnt,
                            &worder, &wkeys, &wsums, &etaken, &etiles})
                b->release(stream);
            for (auto* b : {&rho[0], &rho[1], &press, &scaled, &alpha}) b->release(stream);
            for (auto* b : {&cell[0], &cell[1], &cell[2]}) b->release(stream);
            for (auto* b : {&warm[0], &warm[1]}) b->release(stream);
            fent.release(stream);
            went.release(stream);
            fgv.release(stream);
            wgv.release(stream);
            partials.release(stream);
            stage.release(stream);
            estage.release(stream);
            tape.cpos.release(stream);
            tape.cvel.release(stream);
            tape.cids.release(stream);
            for (auto& r : tape.subs) r->release(stream);
            for (auto& r : spare_records) r->release(stream);
            back.release(stream);
            for (auto* b : {&dmpos, &dmvel, &dcentre, &dfelt}) b->release(stream);
            dmstart.release(stream);
            dwet.release(stream);
            dmcount.release(stream);
            dmtiles.release(stream);
            dmpair.release(stream);
            dmkeys.release(stream);
            rec_rate.release(stream);
            rec_vel.release(stream);
            dwalls.release(stream);
            dwkeys.release(stream);
            dregions.release(stream);
            for (auto* b : {&ddist, &dfar, &ddamping}) b->release(stream);
            dsites.release(stream);
            gslope.release(stream);
            cudaStreamSynchronize(stream);
            drop_solve_graphs();
            drop_substep_graphs();
            for (auto c : cap)
                if (c) cudaStreamDestroy(c);
            if (d_status) cudaFree(d_status);
            if (d_consts) cudaFree(d_consts);
            if (h_status) cudaFreeHost(h_status);
            if (h_reset) cudaFreeHost(h_reset);
            cudaStreamDestroy(stream);
        }
    }

    // ---- settings ----------------------------------------------------------------------------

    static bool valid(const slf_settings& s) {
        auto positive = [](float v) { return std::isfinite(v) && v > 0.0f; };
        bool support = s.support >= 1.5f && s.support <= 4.0f;
        return (s.solver == SLF_SOLVER_WCSPH || s.solver == SLF_SOLVER_DFSPH) && positive(s.spacing) &&
               positive(s.rest_density) && support && s.max_particles > 0 && positive(s.sound_speed) &&
               std::isfinite(s.viscosity) && s.viscosity >= 0.0f && finite3(s.gravity) && s.courant > 0.0f &&
               s.courant <= 1.0f && s.max_substeps > 0 && s.min_iterations <= s.max_iterations &&
               std::isfinite(s.divergence_tolerance) && std::isfinite(s.density_tolerance);
    }

    // rest_mass (src/fluid/mod.rs:694-709)
    float rest_mass() const {
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

    int32_t init(const slf_settings& settings) {
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

    // GroundSites::new (terrain.rs:188-238), in the reference's f32 order
    void build_ground_sites() {
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

    // the terrain regions and ground sites on the device, after a change
    int32_t upload_terrain() {
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

    // per-particle ground slopes of the density pass (null without terrain)
    float4* ground_slopes() {
        if (terrains.empty()) return nullptr;
        if (gslope.ensure(std::max<uint64_t>(n, 1), 0, stream) != SLF_OK) return nullptr;
        return gslope.p;
    }

    static constexpr size_t kMaxTerrainNodes = size_t(1) << 24;  // terrain.rs:9

    // add_terrain's node lattice (terrain.rs:275-283)
    int32_t terrain_nodes(const float* low, const float* high, uint64_t nodes[3]) const {
        if (!finite3(low) || !finite3(high)) return fail(SLF_ERR_NON_FINITE, "non finite value in terrain box");
        if (high[0] <= low[0] || high[1] <= low[1] || high[2] <= low[2])
            return fail(SLF_ERR_OUT_OF_RANGE, "inside out terrain box");
        float step = s.spacing / 2.0f;
        for (int a = 0; a < 3; ++a) nodes[a] = uint64_t(rmin(std::ceil((high[a] - low[a]) / step), 1e7f)) + 1;
        unsigned __int128 total = (unsigned __int128)nodes[0] * nodes[1] * nodes[2];
        if (total > kMaxTerrainNodes) return fail(SLF_ERR_FLUID_FULL, "terrain region holds too many nodes");
        return SLF_OK;
    }

    // add_terrain (terrain.rs:262-302) with distances the caller sampled at the nodes
    int32_t add_terrain(const float* low, const float* high, const float* distances, uint64_t count, uint32_t* out) {
        if (fast()) return fail(SLF_ERR_UNSUPPORTED, "terrain runs with EXACT arithmetic only");
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


    Params params() const {
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

    // viscosity(dt) (step.rs:254-259) and the wall damping (step.rs:282-283)
    StepConsts consts(float dt) const {
        StepConsts c{};
        c.dt = dt;
        c.viscosity = rmin(s.viscosity * s.sound_speed * radius, 0.05f * radius * radius / dt);
        float stable = radius * radius / dt;
        c.wall_viscosity = rmin(1.0f * s.sound_speed * radius, 0.25f * stable);
        c.dt_sq = dt * dt;
        c.mover_damping = rmin(1.0f * s.sound_speed * radius, 0.25f * radius * radius / dt);
        return c;
    }

    Key3 cell_of(F3 p) const {
        return Key3{sat_i32(std::floor(p.x / radius)), sat_i32(std::floor(p.y / radius)),
                    sat_i32(std::floor(p.z / radius))};
    }

    // ---- particles ---------------------------------------------------------------------------

    uint64_t total() const { return n + pend_ids.size(); }
    // FAST list entries keep the index in 26 bits
    static uint64_t index_limit_of(const slf_settings& st) {
        return st.arithmetic == SLF_ARITHMETIC_FAST ? (uint64_t(1) << 26) : UINT64_MAX;
    }
    uint64_t index_limit() const { return index_limit_of(s); }

    int32_t add(uint64_t k, const float* p, const float* v, uint32_t* ids_out) {
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

    // fill_box (src/fluid/mod.rs:493-524)
    int32_t fill_box(const float* low, const float* high, uint64_t* count_out) {
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

    // Moves staged particles onto the device, after the committed ones.
    int32_t flush() {
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

    int32_t ensure_work_buffers() {
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

    bool fast() const { return s.arithmetic == SLF_ARITHMETIC_FAST; }
    // cell-relative positions (always with FAST arithmetic)
    bool rel() const { return s.positions == SLF_POSITIONS_CELL_RELATIVE; }
    int4* cells_of(int slot) const { return rel() ? cell[slot].p : nullptr; }

    // the pair passes of the settings' arithmetic, over the positions of slot a
    // (on: the stream of a graph capture; the world's stream when null)
    void density_pass(const Params& p, int a, const PairLists& fl, const PairLists& wl, float* rh,
                      cudaStream_t on = nullptr) {
        if (!on) on = stream;
        if (fast())
            launch_density_fast(p, fgrid, wgrid, pos[a].p, cells_of(a), dwalls.p, fl, wl, rh, press.p, scaled.p,
                                alpha.p, d_status, on);
        else
            launch_density(p, fgrid, wgrid, pos[a].p, dwalls.p, fl, wl, rh, press.p, scaled.p, alpha.p, d_status,
                           tdev, ground_slopes(), on, mover_dev());
    }
    void force_pass(const Params& p, const PairLists& fl, const PairLists& wl, int a, int b, int nid,
                    cudaStream_t on = nullptr) {
        if (!on) on = stream;
        if (fast())
            launch_wcsph_force_fast(p, d_consts, fl, wl, pos[a].p, cells_of(a), vel[a].p, rho[nid].p, press.p,
                                    scaled.p, dwalls.p, pos[b].p, cells_of(b), vel[b].p, d_status, vel_pre, on);
        else
            launch_wcsph_force(p, d_consts, fl, wl, pos[a].p, vel[a].p, rho[nid].p, press.p, scaled.p, dwalls.p,
                               pos[b].p, vel[b].p, d_status, vel_pre, tdev, terrains.empty() ? nullptr : gslope.p,
                               on, mover_dev());
    }
    // cs, loop: the stream of a graph capture and the while-node handle of its solve loop
    void rate_pass(int which, const Params& p, const PairLists& fl, const PairLists& wl, int a, float4* v, int nid,
                   SolveRec rec = SolveRec{nullptr, nullptr}, cudaStream_t cs = nullptr,
                   unsigned long long loop = 0) {
        cudaStream_t on = cs ? cs : stream;
        if (fast())
            launch_rate_fast(which, rel(), p, d_consts, fl, wl, pos[a].p, v, rho[nid].p, alpha.p, dwalls.p,
                             partials.p, d_status, rec, on, loop);
        else
            launch_rate(which, p, d_consts, fl, wl, pos[a].p, v, rho[nid].p, alpha.p, dwalls.p, partials.p, d_status,
                        rec, on, loop);
    }
    void push_pass(const Params& p, const PairLists& fl, const PairLists& wl, int a, float4* v,
                   float* applied = nullptr, cudaStream_t cs = nullptr, unsigned long long loop = 0) {
        cudaStream_t on = cs ? cs : stream;
        if (fast()) launch_push_fast(rel(), p, d_consts, fl, wl, pos[a].p, v, dwalls.p, d_status, applied, on, loop);
        else launch_push(p, d_consts, fl, wl, pos[a].p, v, dwalls.p, d_status, applied, on, loop);
    }
    bool warm_on() const { return s.warm_start && s.solver == SLF_SOLVER_DFSPH; }
    const float2* warm_in() const { return warm_on() ? warm[cid].p : nullptr; }
    float2* warm_out() { return warm_on() ? warm[1 - cid].p : nullptr; }
    void advance_pass(const Params& p, int a, int b, float4* pre, cudaStream_t on = nullptr) {
        if (!on) on = stream;
        if (rel()) launch_advance_rel(p, d_consts, pos[a].p, cell[a].p, pos[b].p, cell[b].p, vel[b].p, d_status, pre,
                                      on);
        else launch_advance(p, d_consts, pos[a].p, pos[b].p, vel[b].p, d_status, pre, on);
    }
    void stats_pass(const Params& p) {
        if (rel()) launch_state_stats_rel(p, cell[cpos].p, vel[cpos].p, d_status, stream);
        else launch_state_stats(p, pos[cpos].p, vel[cpos].p, d_status, stream);
    }
    void viscous_pass(const Params& p, const PairLists& fl, const PairLists& wl, int a, int b, int nid,
                      cudaStream_t on = nullptr) {
        if (!on) on = stream;
        if (fast())
            launch_viscous_fast(rel(), p, d_consts, fl, wl, pos[a].p, vel[a].p, rho[nid].p, dwalls.p, vel[b].p,
                                on);
        else
            launch_viscous(p, d_consts, fl, wl, pos[a].p, vel[a].p, rho[nid].p, dwalls.p, vel[b].p, on);
    }

    const uint32_t* walk_order() const { return worder_valid ? worder.p : nullptr; }
    // EXACT DFSPH keeps each pair's gradient for the solver check (16 bytes a slot, fluid and
    // walls): the check then gathers a neighbour's velocity only, not its position too
    bool keeps_gradients() const { return SLF_KEEP_GRADIENTS && !fast() && s.solver == SLF_SOLVER_DFSPH; }
    PairLists fluid_lists() const {
        return PairLists{list_cap, fent.p, fcnt.p, walk_order(), keeps_gradients() ? fgv.p : nullptr};
    }
    PairLists wall_lists() const {
        return PairLists{list_cap, went.p, wcnt.p, walk_order(), keeps_gradients() ? wgv.p : nullptr};
    }

    // After a density pass: a list longer than its room leaves the substep to be run again.
    static constexpr int32_t kRetry = -1;
    // The status then holds the failed substep's fields, so the committed state's box and speed
    // are taken again for the rerun's sort.
    int32_t lists_fit() {
        if (h_status->list_max <= list_cap) return SLF_OK;
        list_cap = (uint32_t(h_status->list_max) + h_status->list_max / 4 + 15u) & ~7u;
        SLF_TRY(ensure_work_buffers());
        stats_fresh = false;
        SLF_TRY(refresh_stats());
        return kRetry;
    }

    // ---- coupled bodies (src/fluid/couple.rs, lift.rs) -------------------------------------

    // A body the water and the caller's rigid world share (couple.rs:15-33): its points, frozen
    // water on its own lattice as deep under its surface as the kernel reaches, and its probes,
    // a lattice through its volume for the lift, both in body axes about its centre.
    struct Coupled {
        uint64_t body;
        std::vector<F3> points, probes;
        float probe_spacing = 0.0f;
        F3 center{0, 0, 0}, velocity{0, 0, 0}, moved{0, 0, 0};
        F3 impulse{0, 0, 0}, angular{0, 0, 0};  // the damping's push this step
    };
    std::vector<Coupled> coupled;
    static constexpr size_t kMaxProbes = 4096;  // lift.rs:8
    // the body points of the running step (couple.rs:35-47), sorted, and their device copies
    std::vector<F3> m_start, m_pos, m_vel;
    std::vector<uint32_t> m_own;
    DevBuf<float4> dmpos, dmvel, dcentre, dfelt;
    DevBuf<uint32_t> dmstart, dwet;
    DevBuf<uint32_t> dmcount, dmtiles;
    DevBuf<float4> dmpair;
    DevBuf<int4> dmkeys;
    GridDev mgrid{};
    std::vector<float4> h_felt;

    MoverDev mover_dev() const {
        MoverDev M{};
        if (m_pos.empty()) return M;
        M.count = uint32_t(m_pos.size());
        M.grid = mgrid;
        M.pos = dmpos.p;
        M.vel = dmvel.p;
        return M;
    }

    // couple.rs:453-511: lattice points `spacing` apart inside the shape, no deeper than `reach`
    static int32_t shape_points(int kind, const float dims[3], float spacing, float reach, uint64_t limit,
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

    uint64_t coupled_points() const {
        uint64_t k = 0;
        for (auto& c : coupled) k += c.points.size();
        return k;
    }

    // couple.rs:165-200
    int32_t couple(uint64_t body, int32_t kind, const float dims[3]) {
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

    // couple.rs:203-207
    bool uncouple(uint64_t body) {
        size_t before = coupled.size();
        coupled.erase(std::remove_if(coupled.begin(), coupled.end(), [&](const Coupled& c) { return c.body == body; }),
                      coupled.end());
        return coupled.size() != before;
    }

    static const slf_body_pose* pose_of(const slf_body_pose* poses, uint64_t n, uint64_t body) {
        for (uint64_t k = 0; k < n; ++k)
            if (poses[k].body == body) return &poses[k];
        return nullptr;
    }
    // position.to_dvec3().as_vec3(): the f64 position rounded to f32
    static F3 center_of(const slf_body_pose& p) {
        return F3{float(p.position[0]), float(p.position[1]), float(p.position[2])};
    }
    static F3 f3v(const float* v) { return F3{v[0], v[1], v[2]}; }

    // couple.rs:255-288: body points where the poses say; bodies without a pose are uncoupled
    void place_movers_at(const slf_body_pose* poses, uint64_t npose) {
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

    // couple.rs:291-322: points `elapsed` into the step, sorted by (cell, owner, place), and their
    // device copies and cell table
    int32_t carry_movers(float elapsed) {
        size_t k = m_start.size();
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

    // couple.rs:325-366: the fastest coupled body that may meet the water within dt.  The water's
    // cells are those of the last sort (the reference's grid).
    int32_t fastest_near_water(float dt, float slow, float& most) {
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

    // After a committed WCSPH substep of length dt: what each body's points took, per chunk of 512
    // particles in particle order, added chunk by chunk (step.rs:173-221); the substep's
    // inputs are slot a's positions and velocities and its densities and pressures
    int32_t mover_felt(float dt, const Params& p, int a, int nid) {
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
        h_felt.resize(2 * chunks * bodies);
        SLF_CUDA(cudaMemcpyAsync(h_felt.data(), dfelt.p, h_felt.size() * sizeof(float4), cudaMemcpyDeviceToHost,
                                 stream));
        SLF_TRY(sync());
        for (size_t c = 0; c < chunks; ++c)
            for (size_t b = 0; b < bodies; ++b) {
                const float4& f = h_felt[2 * (c * bodies + b)];
                const float4& t = h_felt[2 * (c * bodies + b) + 1];
                coupled[b].impulse = coupled[b].impulse + F3{f.x, f.y, f.z} * dt;
                coupled[b].angular = coupled[b].angular + F3{t.x, t.y, t.z} * dt;
            }
        return SLF_OK;
    }

    // lift.rs:24-158: what the water does to each coupled body over dt, read as one smooth field
    // around it, from the committed positions and velocities (host copies in p, v)
    struct Lift {
        size_t owner;
        F3 impulse, angular;
        std::vector<uint32_t> near;
    };
    std::vector<Lift> lifts(float dt, const slf_body_pose* poses, uint64_t npose, const std::vector<F3>& P,
                            const std::vector<F3>& V) const {
        F3 g{s.gravity[0], s.gravity[1], s.gravity[2]};
        float grav = length(g);
        F3 up = grav > 0.0f ? (-g) / grav : F3{0.0f, 1.0f, 0.0f};
        float reach = 3.0f * radius;
        float column = radius;
        std::vector<Lift> out;
        for (size_t owner = 0; owner < coupled.size(); ++owner) {
            const Coupled& known = coupled[owner];
            const slf_body_pose* state = pose_of(poses, npose, known.body);
            if (!state) continue;
            F3 center = center_of(*state), lin = f3v(state->linear_velocity), ang = f3v(state->angular_velocity);
            std::vector<std::pair<F3, F3>> probes;
            for (const F3& local : known.probes) {
                F3 arm = rotate(state->rotation, local);
                probes.push_back({arm, lin + cross(ang, arm)});
            }
            F3 low{FLT_MAX, FLT_MAX, FLT_MAX}, high{-FLT_MAX, -FLT_MAX, -FLT_MAX};
            for (auto& pr : probes) {
                low = vmin(low, center + pr.first);
                high = vmax(high, center + pr.first);
            }
            low = low - F3{reach, reach, reach};
            high = high + F3{reach, reach, reach};
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

    // couple.rs:219-248 with the rigid world left to the caller
    int32_t step_with_bodies(float dt, const slf_body_pose* poses, uint64_t npose, slf_report* out,
                             std::vector<slf_body_push>& pushes) {
        pushes.clear();
        if (s.solver != SLF_SOLVER_WCSPH && !coupled.empty())
            return fail(SLF_ERR_INVALID_SETTINGS, "the divergence free solver does not couple yet");
        if (!coupled.empty() && fast()) return fail(SLF_ERR_UNSUPPORTED, "coupled bodies run with EXACT arithmetic only");
        if (tape.on && !coupled.empty()) return fail(SLF_ERR_UNSUPPORTED, "the adjoint takes no coupled bodies");
        place_movers_at(poses, npose);
        int32_t st = step(dt, out);
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
        std::vector<F3> P, V;
        if (n) {
            std::vector<float> hp(3 * n), hv(3 * n);
            SLF_TRY(read_state(hp.data(), hv.data(), n));
            P.resize(n);
            V.resize(n);
            for (uint64_t i = 0; i < n; ++i) {
                P[i] = F3{hp[3 * i], hp[3 * i + 1], hp[3 * i + 2]};
                V[i] = F3{hv[3 * i], hv[3 * i + 1], hv[3 * i + 2]};
            }
        }
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
            std::vector<float> hv(3 * n);
            for (uint64_t i = 0; i < n; ++i) {
                hv[3 * i] = V[i].x;
                hv[3 * i + 1] = V[i].y;
                hv[3 * i + 2] = V[i].z;
            }
            SLF_TRY(write_vec(vel[cpos], hv.data(), n));
            SLF_TRY(sync());
            stats_fresh = false;
        }
        return SLF_OK;
    }

    // ---- walls (src/fluid/boundary.rs) -------------------------------------------------------

    static int32_t check_box(const float* low, const float* high) {
        if (!finite3(low) || !finite3(high)) return fail(SLF_ERR_NON_FINITE, "non finite value in fluid box");
        if (high[0] <= low[0] || high[1] <= low[1] || high[2] <= low[2])
            return fail(SLF_ERR_OUT_OF_RANGE, "inside out fluid box");
        return SLF_OK;
    }

    void cells_in(const float* low, const float* high, int64_t out[3]) const {
        for (int a = 0; a < 3; ++a) {
            float c = rmin(std::round((high[a] - low[a]) / s.spacing), 1e9f);
            out[a] = int64_t(c);
        }
    }

    int32_t check_room(int64_t count) const {
        uint64_t room = s.max_particles > wpos.size() ? s.max_particles - wpos.size() : 0;
        if (index_limit() < UINT64_MAX) room = std::min<uint64_t>(room, index_limit() > wpos.size() ? index_limit() - wpos.size() : 0);
        if (count < 0 || uint64_t(count) > room || wall_next == UINT32_MAX)
            return fail(SLF_ERR_FLUID_FULL, "fluid has no room for more particles");
        return SLF_OK;
    }

    uint32_t add_wall_points(const std::vector<F3>& pts) {
        uint32_t id = wall_next++;
        for (auto& p : pts) {
            wpos.push_back(p);
            wown.push_back(id);
        }
        settle_walls();
        return id;
    }

    int32_t add_box_container(const float* low, const float* high, uint32_t* out) {
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

    int32_t add_wall(const float* low, const float* high, uint32_t* out) {
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

    bool remove_boundary(uint32_t id) {
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

    void update_bounds() {
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

    static uint32_t fbits(float v) {
        uint32_t b;
        std::memcpy(&b, &v, 4);
        return b;
    }

    // settle_walls (boundary.rs:155-178): sort by cell, owner, position bits, index.
    void settle_walls() {
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

    // The cell table of points sorted by cell (keys in order, m = keys.size()): dense over their
    // box while it holds at most 64 cells per occupied one plus 4096 (mod.rs:214-216), else the
    // occupied cells for search; uploaded into dstart / dkeys, described by g.
    int32_t grid_from_keys(const std::vector<Key3>& keys, GridDev& g, DevBuf<uint32_t>& dstart, DevBuf<int4>& dkeys) {
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

    // Uploads the walls and their cell table: dense over the walls' box while it holds at most 64
    // cells per occupied one plus 4096 (mod.rs:214-216), else the occupied cells for search.
    int32_t upload_walls() {
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

    // ---- status --------------------------------------------------------------------------

    // non-finite values in the last passes
    int32_t check_state() const {
        if (h_status->nonfinite) return fail(SLF_ERR_NON_FINITE, "non finite value in fluid particle");
        return SLF_OK;
    }

    int32_t read_status() {
        SLF_CUDA(cudaMemcpyAsync(h_status, d_status, sizeof(Status), cudaMemcpyDeviceToHost, stream));
        return sync();
    }

    // Clears the per-substep fields; the box starts empty.
    static Status fresh_status() {
        Status z{};
        z.cell_lo[0] = z.cell_lo[1] = z.cell_lo[2] = INT32_MAX;
        z.cell_hi[0] = z.cell_hi[1] = z.cell_hi[2] = INT32_MIN;
        return z;
    }
    int32_t reset_status() {
        *h_status = fresh_status();
        SLF_CUDA(cudaMemcpyAsync(d_status, h_status, sizeof(Status), cudaMemcpyHostToDevice, stream));
        return SLF_OK;
    }

    // Box of cells and fastest speed of the committed state.
    int32_t refresh_stats() {
        if (stats_fresh) return SLF_OK;
        SLF_TRY(reset_status());
        Params p = params();
        timed("stats", bytes_per_particle::stats, [&] { stats_pass(p); });
        SLF_TRY(read_status());
        stats_fresh = true;
        return SLF_OK;
    }

    float fastest() const { float v; uint32_t b = h_status->vmax_bits; std::memcpy(&v, &b, 4); return v; }

    // ---- the spatial hash (update_neighbors, src/fluid/mod.rs:540-566) ------------------------

    // Sorts the committed state into slot `to` (pos/vel) and the other id slot, by (cell, id).
    // Needs the committed state's box in the status.  Commits nothing.
    int32_t sort_into(int to) {
        if (n == 0) return SLF_OK;
        SortPlan sp;
        SLF_TRY(plan_sort(sp, false));
        return enqueue_sort(to, sp, stream);
    }

    // What a sort's launches take, fixed on the host before they are queued: the dense cell
    // table's box, the particle range whose destinations are skipped, and whether the lists get a
    // walk order.  Planning also sizes every buffer the sort and the pair passes write, so that
    // the launches can be recorded into a graph (which allocates nothing).
    struct SortPlan {
        int3 lo{}, span{};
        uint32_t volume = 0;
        size_t keys = 0;  // walk-order keys; 0 when the lists keep the particle order
        uint32_t job_lo = 0, job_hi = 0;
    };
    // stable: the table's box is the container's cells joined with the particles' (their own box
    // when that is too large for the table).  Cells are ordered by (x, y, z) over any box that
    // holds them, so the sort's order, and everything after it, is the same over either box.
    int32_t plan_sort(SortPlan& sp, bool stable) {
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
        bool warp_passes = !fast() && s.solver == SLF_SOLVER_WCSPH && n <= kWarpPassMax && terrains.empty() &&
                           m_pos.empty();
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

    // the planned sort's launches on stream `on`
    int32_t enqueue_sort(int to, const SortPlan& sp, cudaStream_t on) {
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

    int32_t update_neighbors() {
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

    int32_t compute_densities() {
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

    // ---- substeps ----------------------------------------------------------------------------

    // one WCSPH substep (step.rs:144-224) from the committed state; commits on success
    int32_t wcsph_substep(float dt, uint32_t& held) {
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

    // solve (dfsph.rs:222-275): Jacobi iterations until the average error is under tolerance.
    // Iterations are queued in batches; the device counts them and turns the launches after
    // the stopping check into no-ops, so the host waits once a batch instead of once an
    // iteration.  A batch is as long as the last solve of the same kind took.
    uint32_t expected_iterations[2] = {2, 2};
    int32_t solve(int which, const Params& p, int a, float4* v, int nid, uint32_t& iterations,
                  SolveRec rec = SolveRec{nullptr, nullptr}) {
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

    // ---- solves as CUDA graphs ----------------------------------------------------------------
    // A solve runs as one graph launch: its resets, the warm push, the first check, then a
    // while node whose body is (push, check).  The check that stops the solve sets the node's
    // condition to 0 on the device, so the host queues the whole substep and waits once, after
    // the advance.  The push bounds the loop at max_iterations + 1 bodies by its own count.
    // Graphs are cached by every value their launches take (slots, buffers, counts, constants),
    // so a cached graph launches exactly what the eager path would.  The eager path stays for
    // the profiler, which times each launch.  A recorded solve (the adjoint's) runs as a graph too
    // but is waited for at once, as its record is copied out by its iteration count.
    static constexpr uint32_t kGraphMaxIterations = 10000;
    static constexpr size_t kGraphCache = 12;
    struct SolveGraph {
        std::vector<uint8_t> key;
        cudaGraphExec_t exec = nullptr;
        uint64_t used = 0;
        uint32_t pre = 0;  // kernels ahead of the loop
    };
    int32_t graph_mode = 2;  // slf_solver_graphs: 0 batched, 1 solves, 2 whole substeps
    std::vector<SolveGraph> solve_graphs;
    uint64_t graph_clock = 0;
    cudaStream_t cap[2] = {nullptr, nullptr};
    uint32_t graph_solves = 0;  // bit w: solve w of the running substep ran as a graph, not yet read

    bool graphs_for(const SolveRec&) const {
        return graph_mode >= 1 && !prof.on && s.max_iterations <= kGraphMaxIterations;
    }
    void drop_solve_graphs() {
        for (auto& g : solve_graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        solve_graphs.clear();
    }
    template <class T> static void key_add(std::vector<uint8_t>& k, const T& v) {
        const uint8_t* b = reinterpret_cast<const uint8_t*>(&v);
        k.insert(k.end(), b, b + sizeof(T));
    }
    static void key_lists(std::vector<uint8_t>& k, const PairLists& l) {
        key_add(k, l.cap);
        key_add(k, l.e);
        key_add(k, l.count);
        key_add(k, l.order);
        key_add(k, l.gv);
    }
    std::vector<uint8_t> solve_key(int which, const Params& p, int a, float4* v, int nid, const PairLists& fl,
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

    // records the solve's launches into a new graph on cap[0] (the loop body on cap[1])
    int32_t capture_solve(int which, const Params& p, int a, float4* v, int nid, const PairLists& fl,
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

    int32_t solve_graph(int which, const Params& p, int a, float4* v, int nid, const PairLists& fl,
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
            if (solve_graphs.size() >= kGraphCache) {
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

    // ---- the whole substep as one graph ------------------------------------------------------
    // In graph mode 2 a substep without a recorded solve or profile is one graph launch: the sort
    // and its walk order, the status reset (a copy from pinned memory), the density pass, then for
    // DFSPH both solves with their device-ended loops, viscosity and the advance, for WCSPH the
    // force and advance pass.  The substep's constants (dt and
    // what follows from it) are read from device memory, written by one launch ahead of the
    // graph, so a graph holds across substeps whose dt changes.  The cell table's box is the
    // container's (plan_sort, stable), so slot rotation alone (3 position slots x 2 id slots)
    // gives the 6 graphs of a steady run.  Graphs are cached by a key of every value their
    // launches take and recorded the first time a key is met, until two graphs leave the cache
    // having run once: from then on (a scene whose count changes every tick: flows, a domain) a
    // key is recorded the second time it is met, and keys met once run the eager launches.
    struct SubstepGraph {
        std::vector<uint8_t> key;
        cudaGraphExec_t exec = nullptr;
        uint64_t used = 0;
        uint64_t runs = 0;
        uint32_t outside = 0;  // kernels outside the solve loops
    };
    std::vector<SubstepGraph> substep_graphs;
    std::vector<std::vector<uint8_t>> substep_seen;  // keys met once, oldest first
    uint64_t graph_substeps = 0;                     // substeps run as one graph launch
    uint32_t unused_graphs = 0;                      // graphs evicted after one run
    static constexpr uint32_t kUnusedGraphs = 2;     // ... after which keys wait for a second sighting

    bool whole_substeps() const {
        // (the adjoint's recomputed substeps, which redirect the sort and record velocities, launch
        // eagerly)
        return graph_mode >= 2 && !prof.on && s.max_iterations <= kGraphMaxIterations && skip_job < 0 &&
               terrains.empty() && m_pos.empty() && n > 0 && !sort_dest && !vel_pre;
    }
    void drop_substep_graphs() {
        for (auto& g : substep_graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        substep_graphs.clear();
        substep_seen.clear();
        unused_graphs = 0;
    }
    std::vector<uint8_t> substep_key(const Params& p, int a, int b, int nid, const SortPlan& sp) {
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

    // records the substep's launches into g.exec (the solve loops' bodies on cap[1])
    int32_t capture_substep(const Params& p, int a, int b, int nid, const SortPlan& sp, SubstepGraph& g) {
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

    // Runs the planned substep as one graph launch when its graph is cached or recorded now;
    // ran = false leaves the substep to the eager launches.
    int32_t substep_graph(float dt, const Params& p, int a, int b, int nid, const SortPlan& sp, bool& ran) {
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

    // After solves that ran as graphs (status read back): their iteration counts, their loop
    // kernels in the launch count, and the checks the batched path makes per solve (the lists'
    // room, the stop flag).  its[w] is set for each solve w that ran.
    int32_t finish_graph_solves(uint32_t its[2]) {
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

    // The launches of a solve after its stopping check did nothing; their profile entries
    // go under "solver_idle" so the kernels' averages hold only launches that worked.
    void relabel_idle(size_t first, const std::vector<int>& kinds, uint32_t iterations) {
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

    // a solve's records land here, max_iterations + 1 slots, before they are kept
    DevBuf<float> rec_rate;
    DevBuf<float4> rec_vel;

    // Records are sized for a quarter more iterations than any solve has recorded yet, so the
    // records a later tape reuses seldom grow: a new device allocation in the middle of a taped
    // run costs far more than the substep.
    uint32_t record_room = 0;
    int32_t keep_record(uint32_t its, DevBuf<float>& rates, DevBuf<float4>& vels) {
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

    // one DFSPH substep (dfsph.rs:79-103) from the committed state; commits on success.  With
    // `rec`, the solves are recorded for the adjoint (the same batched launches, the slot of
    // each check taken from the device's iteration count).
    int32_t dfsph_substep(float dt, uint32_t& held, uint32_t& iterations, DfsphRecord* rec = nullptr) {
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
    uint32_t last_iterations[2] = {0, 0};

    // step (step.rs:58-90), recorded when a tape is on
    int32_t step(float dt, slf_report* out) {
        if (!tape.on) return step_untaped(dt, out);
        SLF_TRY(flush());
        if (n != tape.n || has_domain || !flows.empty())
            return fail(SLF_ERR_UNSUPPORTED, "the particles changed while a tape was recording");
        tape.steps.emplace_back();
        tape_step = &tape.steps.back();
        size_t recorded = tape.subs.size();
        int32_t st = step_untaped(dt, out);
        tape_step = nullptr;
        if (st != SLF_OK) {
            tape.steps.pop_back();
            drop_records(recorded);
            return st;
        }
        if (tape.every && tape.steps.size() % tape.every == 0) SLF_TRY(checkpoint());
        return SLF_OK;
    }

    // ---- the adjoint ---------------------------------------------------------------------------

    int32_t tape_begin(uint32_t every) {
        if (rel()) return fail(SLF_ERR_UNSUPPORTED, "the adjoint runs on absolute positions only");
        if (!terrains.empty()) return fail(SLF_ERR_UNSUPPORTED, "the adjoint takes no terrain");
        if (warm_on()) return fail(SLF_ERR_UNSUPPORTED, "the adjoint runs on cold-started solves only");
        SLF_TRY(flush());
        tape.on = true;
        tape.every = every;
        tape.n = n;
        tape.steps.clear();
        tape.ckpt_step.clear();
        drop_records(0);
        return every ? checkpoint() : SLF_OK;
    }

    // gives the recorded substeps from the keep-th on back to the spares
    void drop_records(size_t keep) {
        while (tape.subs.size() > keep) {
            spare_records.push_back(std::move(tape.subs.back()));
            tape.subs.pop_back();
        }
    }

    // a new substep record holding the committed state, for a tape with every == 0
    int32_t record_begin(float dt) {
        auto sub = new_record();
        sub->dt = dt;
        SLF_TRY(sub->pos.ensure(n, 0, stream));
        SLF_TRY(sub->vel.ensure(n, 0, stream));
        SLF_TRY(sub->ids.ensure(n, 0, stream));
        SLF_TRY(save_state(sub->pos.p, sub->vel.p, sub->ids.p));
        tape.subs.push_back(std::move(sub));
        return SLF_OK;
    }

    // the tape's buffers (records, checkpoints, solver scratch) stay for the next tape
    int32_t tape_end() {
        tape.on = false;
        tape.steps.clear();
        tape.ckpt_step.clear();
        drop_records(0);
        return sync();
    }

    // the committed state becomes checkpoint number ckpt_step.size()
    int32_t checkpoint() {
        size_t c = tape.ckpt_step.size(), m = n;
        SLF_TRY(tape.cpos.ensure((c + 1) * m, c * m, stream));
        SLF_TRY(tape.cvel.ensure((c + 1) * m, c * m, stream));
        SLF_TRY(tape.cids.ensure((c + 1) * m, c * m, stream));
        SLF_TRY(save_state(tape.cpos.p + c * m, tape.cvel.p + c * m, tape.cids.p + c * m));
        tape.ckpt_step.push_back(tape.steps.size());
        return SLF_OK;
    }

    int32_t save_state(float4* p, float4* v, uint32_t* id) {
        if (!n) return SLF_OK;
        SLF_CUDA(cudaMemcpyAsync(p, pos[cpos].p, n * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
        SLF_CUDA(cudaMemcpyAsync(v, vel[cpos].p, n * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
        SLF_CUDA(cudaMemcpyAsync(id, ids[cid].p, n * 4, cudaMemcpyDeviceToDevice, stream));
        return SLF_OK;
    }

    int32_t load_state(const float4* p, const float4* v, const uint32_t* id) {
        if (n) {
            SLF_CUDA(cudaMemcpyAsync(pos[cpos].p, p, n * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
            SLF_CUDA(cudaMemcpyAsync(vel[cpos].p, v, n * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
            SLF_CUDA(cudaMemcpyAsync(ids[cid].p, id, n * 4, cudaMemcpyDeviceToDevice, stream));
        }
        stats_fresh = false;
        lists_valid = false;
        return refresh_stats();
    }

    int32_t substep_retrying(float dt) {
        uint32_t held = 0, its = 0;
        auto once = [&] { return s.solver == SLF_SOLVER_WCSPH ? wcsph_substep(dt, held) : dfsph_substep(dt, held, its); };
        int32_t st = once();
        if (st == kRetry) st = once();
        if (st == kRetry) st = fail(SLF_ERR_CUDA, "neighbour lists outgrew their room twice");
        return st;
    }

    // The sort and density pass of a DFSPH substep from the committed state, without the
    // solves: the lists, factors and densities the adjoint of a recorded substep reads.  The
    // sort's destinations go to sort_dest.  Commits nothing; returns the slots used.
    int32_t dfsph_replay(float dt, int& a, int& nid) {
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

    // step_backward: reverse over the taped steps, one checkpoint segment at a time.
    int32_t step_backward(const float* dpos, const float* dvel, uint64_t k, float* dpos0, float* dvel0,
                          slf_param_grads* out) {
        if (!tape.on || tape.steps.empty()) return fail(SLF_ERR_OUT_OF_RANGE, "no steps recorded");
        SLF_TRY(flush());
        if (k != n || n != tape.n) return fail(SLF_ERR_INVALID_ARGUMENT, "n must equal slf_len()");
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
            SLF_TRY(save_state(spos.p, svel.p, sids.p));
            SLF_CUDA(cudaMemcpyAsync(srho.p, rho[cid].p, n * 4, cudaMemcpyDeviceToDevice, stream));
            SLF_TRY(write_vec(xo, dpos, n));
            SLF_TRY(write_vec(vo, dvel, n));
            // the adjoint of the substep whose forward state sits in slots a (sorted positions)
            // and nid (densities), its constants in d_consts: (xo, vo) after it -> (xp, vp) before
            auto adjoint_substep = [&](float dt, int a, int nid, const DfsphRecord& rec) -> int32_t {
                Params p = params();
                SLF_CUDA(cudaMemsetAsync(grads.p, 0, kGradSlots * sizeof(double), stream));
                PairLists fl = fluid_lists(), wl = wall_lists();
                bool packed = !fast();
                if (s.solver == SLF_SOLVER_WCSPH) {
                    launch_adjoint_wcsph(p, d_consts, fl, wl, packed, pos[a].p, vel[a].p, rho[nid].p, press.p,
                                         scaled.p, dwalls.p, pre.p, dest.p, xo.p, vo.p, ab.p, xb.p, vb.p, rb.p, xp.p,
                                         vp.p, grads.p, stream);
                } else {
                    // advance, density solve, viscosity, divergence solve, factors, densities,
                    // sort: the substep's steps backwards
                    timed("adj_advance", 0.0, [&] {
                        launch_adj_advance_dfsph(p, d_consts, rec.pre.p, xo.p, vo.p, xb.p, vb.p, stream);
                    });
                    SLF_CUDA(cudaMemsetAsync(rb.p, 0, n * 4, stream));
                    SLF_CUDA(cudaMemsetAsync(abar.p, 0, n * 4, stream));
                    for (uint32_t it = rec.den_n; it-- > 0;) {
                        for (int part = 1; part <= 2; ++part)
                            timed(part == 1 ? "adj_kappa_density" : "adj_push_density", 0.0, [&] {
                                launch_adj_iteration(1, p, d_consts, fl, wl, packed, pos[a].p, dwalls.p, vb.p,
                                                     rec.den_rate.p + size_t(it) * n, alpha.p, rho[nid].p,
                                                     rec.den_vel.p + size_t(it) * n, kw.p, vr.p, abar.p, rb.p,
                                                     vp.p, xb.p, stream, part);
                            });
                        std::swap(vb, vp);
                    }
                    timed("adj_viscosity", 0.0, [&] {
                        launch_adj_viscosity(p, d_consts, fl, wl, packed, pos[a].p, rec.va.p, rho[nid].p, zeros.p,
                                             dwalls.p, vb.p, ab.p, xb.p, rb.p, grads.p, stream);
                    });
                    for (uint32_t it = rec.div_n; it-- > 0;) {
                        for (int part = 1; part <= 2; ++part)
                            timed(part == 1 ? "adj_kappa_divergence" : "adj_push_divergence", 0.0, [&] {
                                launch_adj_iteration(0, p, d_consts, fl, wl, packed, pos[a].p, dwalls.p, vb.p,
                                                     rec.div_rate.p + size_t(it) * n, alpha.p, rho[nid].p,
                                                     rec.div_vel.p + size_t(it) * n, kw.p, vr.p, abar.p, rb.p,
                                                     vp.p, xb.p, stream, part);
                            });
                        std::swap(vb, vp);
                    }
                    timed("adj_factors_density", 0.0, [&] {
                        launch_adj_factors_density(p, fl, wl, packed, pos[a].p, dwalls.p, alpha.p, abar.p, gt.p,
                                                   rb.p, xb.p, stream);
                    });
                    timed("adj_unsort", 0.0, [&] { launch_adj_unsort(uint32_t(n), dest.p, xb.p, vb.p, xp.p, vp.p, stream); });
                }
                double g[kGradSlots];
                SLF_CUDA(cudaMemcpyAsync(g, grads.p, sizeof(g), cudaMemcpyDeviceToHost, stream));
                SLF_TRY(sync());
                accumulate_param_grads(dt, g, pg);
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
                    SLF_TRY(load_state(sub.pos.p, sub.vel.p, sub.ids.p));
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
                for (size_t c = tape.ckpt_step.size(); c-- > 0;) {
                    size_t b = tape.ckpt_step[c];
                    size_t e = c + 1 < tape.ckpt_step.size() ? tape.ckpt_step[c + 1] : tape.steps.size();
                    if (b >= e) continue;
                    std::vector<float> dts;
                    for (size_t t = b; t < e; ++t) dts.insert(dts.end(), tape.steps[t].begin(), tape.steps[t].end());
                    while (segsubs.size() < dts.size()) segsubs.push_back(new_record());
                    SLF_TRY(load_state(tape.cpos.p + c * n, tape.cvel.p + c * n, tape.cids.p + c * n));
                    for (size_t q = 0; q < dts.size(); ++q) {
                        SubRecord& sub = *segsubs[q];
                        sub.dt = dts[q];
                        SLF_TRY(sub.pos.ensure(n, 0, stream));
                        SLF_TRY(sub.vel.ensure(n, 0, stream));
                        SLF_TRY(sub.ids.ensure(n, 0, stream));
                        SLF_TRY(save_state(sub.pos.p, sub.vel.p, sub.ids.p));
                        uint32_t held = 0, its = 0;
                        int32_t rs;
                        if (s.solver == SLF_SOLVER_WCSPH) {
                            rs = wcsph_substep(dts[q], held);
                            if (rs == kRetry) rs = wcsph_substep(dts[q], held);
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
            SLF_TRY(load_state(spos.p, svel.p, sids.p));
            SLF_CUDA(cudaMemcpyAsync(rho[cid].p, srho.p, n * 4, cudaMemcpyDeviceToDevice, stream));
            return sync();
        };
        st = run();
        sync();
        if (st == SLF_OK && out) *out = pg;
        return st;
    }

    // The substep's sensitivities to its derived constants, taken back to the settings:
    // nu = min(viscosity c r, 0.05 r^2 / dt) (step.rs:254-259), nu_w = min(c r, 0.25 r^2 / dt)
    // (step.rs:282-283), B = rest c^2 / 7 (step.rs:149); the branch the substep took decides.
    void accumulate_param_grads(float dt, const double* g, slf_param_grads& pg) const {
        double r = radius, c = s.sound_speed, visc = s.viscosity;
        bool nu_free = double(s.viscosity) * c * r < 0.05 * r * r / dt;
        bool nuw_free = c * r < 0.25 * r * r / dt;
        if (nu_free) {
            pg.viscosity += g[kGradViscosity] * c * r;
            pg.sound_speed += g[kGradViscosity] * visc * r;
        }
        if (nuw_free) pg.sound_speed += g[kGradWallViscosity] * r;
        pg.sound_speed += g[kGradStiffness] * 2.0 * double(s.rest_density) * c / 7.0;
        for (int a = 0; a < 3; ++a) pg.gravity[a] += g[kGradGravity + a];
    }

    int32_t step_untaped(float dt, slf_report* out) {
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
                    if (tape_step) tape_step->push_back(small);
                    if (tape_step && tape.every == 0) SLF_TRY(record_begin(small));
                    if (!coupled.empty()) SLF_TRY(carry_movers(small * float(i)));
                    int32_t st = wcsph_substep(small, held);
                    if (st == kRetry) st = wcsph_substep(small, held);
                    if (st == kRetry) st = fail(SLF_ERR_CUDA, "neighbour lists outgrew their room twice");
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
                    if (tape_step) tape_step->push_back(small);
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

    // Keeps, in order, the particles inside the box (drain = 0) or outside it (drain = 1);
    // `removed` counts the others.
    int32_t keep_where(F3 low, F3 high, int drain, uint32_t& removed) {
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

    // keep_in_domain (mod.rs:451-486)
    int32_t keep_in_domain(uint32_t& lost) {
        lost = 0;
        if (!has_domain) return SLF_OK;
        return keep_where(dlow, dhigh, 0, lost);
    }

    // ---- emitters and drains (src/fluid/flow.rs) ---------------------------------------------

    struct FlowBox {
        uint32_t id;
        F3 low, high;
        bool emitter;
        F3 velocity;
    };
    std::vector<FlowBox> flows;
    uint32_t flow_next = 0;
    DevBuf<uint32_t> etaken, etiles;
    DevBuf<float4> estage;

    // add_flow (flow.rs:115-139), add_emitter (:86-99), add_drain (:104-106)
    int32_t add_flow(const float* low, const float* high, bool emitter, const float* velocity, uint32_t* out) {
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

    // remove_flow (flow.rs:109-113)
    bool remove_flow(uint32_t id) {
        size_t before = flows.size();
        flows.erase(std::remove_if(flows.begin(), flows.end(), [&](const FlowBox& f) { return f.id == id; }),
                    flows.end());
        return flows.size() != before;
    }

    // Rust's `f as i64`: saturating, NaN to 0
    static int64_t as_i64(float v) {
        if (std::isnan(v)) return 0;
        if (v >= 9.2233720e18f) return INT64_MAX;
        if (v <= -9.2233720e18f) return INT64_MIN;
        return int64_t(v);
    }

    // run_flows (flow.rs:144-231): drains first, then emitters, each in the order they were
    // added.  An emitter whose lattice would hold more than 2^30 slots is refused (the reference
    // allocates one flag per slot, up to 4096^3).
    int32_t run_flows(uint32_t& emitted, uint32_t& drained) {
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

    // ---- snapshots (src/fluid/save.rs) ---------------------------------------------------------

    // save_snapshot (save.rs:18-73): the SLFL version 3 bytes of the current state, particles in
    // their current order; no coupled bodies or terrains exist on this path.
    int32_t save_snapshot(std::vector<uint8_t>& out) {
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

    // load_snapshot (save.rs:79-181) into a fresh world: untrusted bytes, checked in the
    // reference's order; the library's own settings fields come from `lib`.
    int32_t load_snapshot(const uint8_t* data, size_t size, const slf_settings& lib) {
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

    // ---- read-outs -------------------------------------------------------------------------

    // packs xyz on the device and copies 12 bytes a particle straight into the caller's buffer
    int32_t read_vec(const DevBuf<float4>& b, float* out, uint64_t k) {
        if (!k) return SLF_OK;
        SLF_TRY(stage.ensure(3 * k, 0, stream));
        launch_pack3(uint32_t(k), b.p, stage.p, stream);
        SLF_CUDA(cudaMemcpyAsync(out, stage.p, k * 12, cudaMemcpyDeviceToHost, stream));
        return sync();
    }

    // the committed positions as xyz triples (cell-relative ones rebuilt in double, rounded once)
    int32_t read_positions(float* out, uint64_t k) {
        if (!rel()) return read_vec(pos[cpos], out, k);
        if (!k) return SLF_OK;
        SLF_TRY(stage.ensure(3 * k, 0, stream));
        launch_from_relative(params(), uint32_t(k), pos[cpos].p, cell[cpos].p, stage.p, stream);
        SLF_CUDA(cudaMemcpyAsync(out, stage.p, k * 12, cudaMemcpyDeviceToHost, stream));
        return sync();
    }

    int32_t write_vec(DevBuf<float4>& b, const float* in, uint64_t k) {
        if (!k) return SLF_OK;
        SLF_TRY(stage.ensure(3 * k, 0, stream));
        SLF_CUDA(cudaMemcpyAsync(stage.p, in, k * 12, cudaMemcpyHostToDevice, stream));
        launch_unpack3(uint32_t(k), stage.p, b.p, stream);
        return SLF_OK;
    }

    // Uploads the caller's state into a free slot, checking it on the device as it unpacks and
    // folding the box and speed the next step needs, then waits once: a state with a non finite
    // value is refused and the committed one stays.
    int32_t write_state(const float* p, const float* v, uint64_t k) {
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

    // positions and velocities into the caller's buffers with one wait
    int32_t read_state(float* p, float* v, uint64_t k) {
        if (!k) return SLF_OK;
        SLF_TRY(stage.ensure(6 * k, 0, stream));
        if (rel()) launch_from_relative(params(), uint32_t(k), pos[cpos].p, cell[cpos].p, stage.p, stream);
        else launch_pack3(uint32_t(k), pos[cpos].p, stage.p, stream);
        launch_pack3(uint32_t(k), vel[cpos].p, stage.p + 3 * k, stream);
        SLF_CUDA(cudaMemcpyAsync(p, stage.p, k * 12, cudaMemcpyDeviceToHost, stream));
        SLF_CUDA(cudaMemcpyAsync(v, stage.p + 3 * k, k * 12, cudaMemcpyDeviceToHost, stream));
        return sync();
    }

    template <class T> int32_t read_plain(const DevBuf<T>& b, T* out, uint64_t k) {
        if (k) {
            SLF_CUDA(cudaMemcpyAsync(out, b.p, k * sizeof(T), cudaMemcpyDeviceToHost, stream));
            SLF_CUDA(cudaStreamSynchronize(stream));
        }
        return SLF_OK;
    }

    int32_t lists(bool walls, uint32_t* start, uint64_t start_len, uint32_t* items, uint64_t cap, uint64_t* len) {
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

    uint64_t state_hash_host(const std::vector<uint32_t>& id, const std::vector<float>& p,
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
};

void set_last_error(const std::string& message) { g_error = message; }

}  // namespace slf

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
