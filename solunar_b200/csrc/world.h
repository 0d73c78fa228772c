// world.h -- the host side of the library: FluidWorld's state owner (struct World), shared by
// the world_*.cpp units that define its methods and by capi.cpp, the C ABI.
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
#pragma once
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

inline thread_local std::string g_error;

inline int32_t fail(int32_t code, const std::string& msg) {
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
        DevBuf<float2> warm;  // warm starts: the impulses the solves started from, sorted
        uint32_t div_n = 0, den_n = 0;
        void release(cudaStream_t st) {
            for (auto* b : {&div_vel, &den_vel, &va, &pre}) b->release(st);
            div_rate.release(st);
            den_rate.release(st);
            warm.release(st);
        }
    };
    // A substep recorded as it ran (tapes that checkpoint every substep's record): the state
    // before it and its solver record.
    struct SubRecord {
        float dt = 0.0f;
        DevBuf<float4> pos, vel;
        DevBuf<uint32_t> ids;
        DevBuf<int4> cells;  // cell-relative positions: the cells of pos's offsets
        DevBuf<float2> warm;  // warm starts: each particle's impulses before the substep
        DfsphRecord rec;
        // A substep that a checkpoint segment ran again keeps what its adjoint reads, so the
        // segment's reverse sweep runs no substep a third time: WCSPH the sorted state, densities
        // and pressures, the sort's destinations, the pre-clamp velocities, the ground slopes,
        // the walk order and both neighbour lists (which change places with the world's); DFSPH
        // the sorted positions, densities and factors, the sort's destinations, the walk order
        // and both lists with their kept gradients (written there by the substep's own density
        // pass), beside its solver record.
        bool kept = false;
        bool ordered = false;  // the lists walk rows in `order`
        uint32_t cap = 0;      // the lists' room a row
        DevBuf<float4> spos, svel, pre, slope;
        DevBuf<int4> scells;
        DevBuf<float> rho, press, scaled, alpha;
        DevBuf<uint32_t> dest, order, fcnt, wcnt;
        DevBuf<uint2> fent, went;
        DevBuf<float4> fgv, wgv;
        // With coupled bodies (tapes that record every substep): the body points the substep
        // met, with their cell table, and the sound speed the step ran at, `raised` when a fast
        // body set it above the settings' (the settings' then take no derivative from it).
        uint32_t mcount = 0;
        GridDev mgrid{};
        DevBuf<float4> mpos, mvel;
        DevBuf<uint32_t> mstart;
        DevBuf<int4> mkeys;
        float sound = 0.0f;
        bool raised = false;
        void release(cudaStream_t st) {
            pos.release(st);
            vel.release(st);
            ids.release(st);
            cells.release(st);
            warm.release(st);
            rec.release(st);
            for (auto* b : {&spos, &svel, &pre, &slope}) b->release(st);
            scells.release(st);
            for (auto* b : {&rho, &press, &scaled, &alpha}) b->release(st);
            for (auto* b : {&dest, &order, &fcnt, &wcnt}) b->release(st);
            fent.release(st);
            went.release(st);
            fgv.release(st);
            wgv.release(st);
            for (auto* b : {&mpos, &mvel}) b->release(st);
            mstart.release(st);
            mkeys.release(st);
            mcount = 0;
            kept = false;
        }
    };
    // After a WCSPH substep of a segment's replay (its sort writing `sub.dest`, its advance
    // `sub.pre`): the substep's forward into `sub` (SubRecord::kept).
    int32_t keep_wcsph_substep(SubRecord& sub);
    // A DFSPH substep of a segment's replay into `sub`: its lists and counts change places with
    // the world's for the substep (the density pass writes them into the record, so the solves'
    // graphs see the same buffers each time the record comes round), its sort writes `sub.dest`;
    // then the sorted positions, densities, factors and walk order are copied.
    int32_t kept_dfsph_substep(float dt, SubRecord& sub);
    void swap_lists(SubRecord& sub);
    // The device buffers a WCSPH checkpoint segment's records take, at the current size and list
    // room, so that the backward allocates nothing (slf_tape_begin reserves a segment of them).
    int32_t reserve_kept(SubRecord& sub);

    // ---- the tape of slf_tape_begin: checkpoints and the substep lengths of each step ----
    struct Tape {
        bool on = false;
        uint32_t every = 1;
        uint64_t n = 0;
        std::vector<std::vector<float>> steps;  // substep lengths of each recorded step
        size_t count = 0;                       // substeps recorded so far
        std::vector<size_t> ckpt_sub;           // checkpoint c = the state before substep ckpt_sub[c]
        DevBuf<float4> cpos, cvel;              // [c][n]
        DevBuf<uint32_t> cids;
        DevBuf<int4> ccells;                    // cell-relative positions: [c][n]
        DevBuf<float2> cwarm;                   // warm starts: [c][n]
        std::vector<std::unique_ptr<SubRecord>> subs;  // every == 0: each substep's record
        bool keep_segments = false;  // WCSPH checkpoint segments keep each substep's forward
    } tape;
    // Records of finished tapes and segments, kept with their device buffers for the next ones:
    // the rounds of an optimisation loop then record without allocating (tens of GB at a
    // million particles, whose first allocation costs far more than the steps).
    std::vector<std::unique_ptr<SubRecord>> spare_records;
    // scratch of slf_step_backward
    struct BackScratch {
        DevBuf<float4> spos, svel, xo, vo, xp, vp, ab, xb, vb, pre, gt, kw, vr;
        DevBuf<uint32_t> sids, dest;
        DevBuf<int4> scells;
        DevBuf<float> srho, rb, abar, zeros;
        DevBuf<double> grads;
        // warm starts: the world's impulses, put back at the end; the adjoint of the impulses
        // each particle's solves leave (after the substep; before it)
        DevBuf<float2> swarm, appbar, appbar_out;
        void release(cudaStream_t s) {
            scells.release(s);
            for (auto* b : {&swarm, &appbar, &appbar_out}) b->release(s);
            for (auto* b : {&spos, &svel, &xo, &vo, &xp, &vp, &ab, &xb, &vb, &pre, &gt, &kw, &vr}) b->release(s);
            for (auto* b : {&srho, &rb, &abar, &zeros}) b->release(s);
            sids.release(s);
            dest.release(s);
            grads.release(s);
        }
    } back;
    std::unique_ptr<SubRecord> new_record();
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

    int32_t sync();

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
            for (auto* b : {&lkeep, &lat, &lidx, &ltiles}) b->release(stream);
            for (auto* b : {&dmcur_start, &dmcur_vel, &dmnext_start, &dmnext_vel, &dimpulse}) b->release(stream);
            for (auto* b : {&dmlin, &dmslot, &dmmembers, &dmtable, &dmtable_tiles}) b->release(stream);
            lpv.release(stream);
            lboxes.release(stream);
            partials.release(stream);
            stage.release(stream);
            estage.release(stream);
            tape.cpos.release(stream);
            tape.cvel.release(stream);
            tape.cids.release(stream);
            tape.ccells.release(stream);
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

    static bool valid(const slf_settings& s);

    // rest_mass (src/fluid/mod.rs:694-709)
    float rest_mass() const;

    int32_t init(const slf_settings& settings);

    // GroundSites::new (terrain.rs:188-238), in the reference's f32 order
    void build_ground_sites();

    // the terrain regions and ground sites on the device, after a change
    int32_t upload_terrain();

    // per-particle ground slopes of the density pass (null without terrain)
    float4* ground_slopes();

    static constexpr size_t kMaxTerrainNodes = size_t(1) << 24;  // terrain.rs:9

    // add_terrain's node lattice (terrain.rs:275-283)
    int32_t terrain_nodes(const float* low, const float* high, uint64_t nodes[3]) const;

    // add_terrain (terrain.rs:262-302) with distances the caller sampled at the nodes
    int32_t add_terrain(const float* low, const float* high, const float* distances, uint64_t count, uint32_t* out);


    Params params() const;

    // viscosity(dt) (step.rs:254-259) and the wall damping (step.rs:282-283)
    StepConsts consts(float dt) const;

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

    int32_t add(uint64_t k, const float* p, const float* v, uint32_t* ids_out);

    // fill_box (src/fluid/mod.rs:493-524)
    int32_t fill_box(const float* low, const float* high, uint64_t* count_out);

    // Moves staged particles onto the device, after the committed ones.
    int32_t flush();

    int32_t ensure_work_buffers();

    bool fast() const { return s.arithmetic == SLF_ARITHMETIC_FAST; }
    // cell-relative positions (always with FAST arithmetic)
    bool rel() const { return s.positions == SLF_POSITIONS_CELL_RELATIVE; }
    int4* cells_of(int slot) const { return rel() ? cell[slot].p : nullptr; }

    // the pair passes of the settings' arithmetic, over the positions of slot a
    // (on: the stream of a graph capture; the world's stream when null)
    void density_pass(const Params& p, int a, const PairLists& fl, const PairLists& wl, float* rh,
                      cudaStream_t on = nullptr);
    void force_pass(const Params& p, const PairLists& fl, const PairLists& wl, int a, int b, int nid,
                    cudaStream_t on = nullptr);
    // cs, loop: the stream of a graph capture and the while-node handle of its solve loop
    void rate_pass(int which, const Params& p, const PairLists& fl, const PairLists& wl, int a, float4* v, int nid,
                   SolveRec rec = SolveRec{nullptr, nullptr}, cudaStream_t cs = nullptr,
                   unsigned long long loop = 0);
    void push_pass(const Params& p, const PairLists& fl, const PairLists& wl, int a, float4* v,
                   float* applied = nullptr, cudaStream_t cs = nullptr, unsigned long long loop = 0);
    bool warm_on() const { return s.warm_start && s.solver == SLF_SOLVER_DFSPH; }
    const float2* warm_in() const { return warm_on() ? warm[cid].p : nullptr; }
    float2* warm_out() { return warm_on() ? warm[1 - cid].p : nullptr; }
    void advance_pass(const Params& p, int a, int b, float4* pre, cudaStream_t on = nullptr);
    void stats_pass(const Params& p) {
        if (rel()) launch_state_stats_rel(p, cell[cpos].p, vel[cpos].p, d_status, stream);
        else launch_state_stats(p, pos[cpos].p, vel[cpos].p, d_status, stream);
    }
    void viscous_pass(const Params& p, const PairLists& fl, const PairLists& wl, int a, int b, int nid,
                      cudaStream_t on = nullptr);

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
    int32_t lists_fit();

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
    // Carrying the points on the device (a step whose points stay within a dense cell box of
    // modest volume): the step's box, the points in their current order (starts with the owner
    // bits in w, velocities), the next order, and the sort's scratch; the table is the grid's.
    // the damping impulse and its torque each body took so far this step ([2 b], [2 b + 1])
    DevBuf<float4> dimpulse;
    bool mdevice = false;
    int3 mlow{}, mspan{};
    uint32_t mvolume = 0;
    DevBuf<float4> dmcur_start, dmcur_vel, dmnext_start, dmnext_vel;
    DevBuf<uint32_t> dmlin, dmslot, dmmembers, dmtable, dmtable_tiles;
    DevBuf<uint32_t> dmcount, dmtiles;
    DevBuf<float4> dmpair;
    DevBuf<int4> dmkeys;
    GridDev mgrid{};

    MoverDev mover_dev() const;

    // couple.rs:453-511: lattice points `spacing` apart inside the shape, no deeper than `reach`
    static int32_t shape_points(int kind, const float dims[3], float spacing, float reach, uint64_t limit,
                                std::vector<F3>& out);

    uint64_t coupled_points() const;

    // couple.rs:165-200
    int32_t couple(uint64_t body, int32_t kind, const float dims[3]);

    // couple.rs:203-207
    bool uncouple(uint64_t body);

    static const slf_body_pose* pose_of(const slf_body_pose* poses, uint64_t n, uint64_t body);
    // position.to_dvec3().as_vec3(): the f64 position rounded to f32
    static F3 center_of(const slf_body_pose& p) {
        return F3{float(p.position[0]), float(p.position[1]), float(p.position[2])};
    }
    static F3 f3v(const float* v) { return F3{v[0], v[1], v[2]}; }

    // couple.rs:255-288: body points where the poses say; bodies without a pose are uncoupled
    void place_movers_at(const slf_body_pose* poses, uint64_t npose);

    // couple.rs:291-322: points `elapsed` into the step, sorted by (cell, owner, place), and their
    // device copies and cell table
    // the points at `elapsed` of the step's substeps, `last` the elapsed time of its last one
    int32_t carry_movers(float elapsed, float last);
    // at the step's first substep: the cell box the points reach over the step (their cells at
    // its first and last substeps: each moves on a line), and whether the device carries them
    int32_t plan_movers(float last);

    // couple.rs:325-366: the fastest coupled body that may meet the water within dt.  The water's
    // cells are those of the last sort (the reference's grid).
    int32_t fastest_near_water(float dt, float slow, float& most);

    // After a committed WCSPH substep of length dt: what each body's points took, per chunk of 512
    // particles in particle order, added chunk by chunk (step.rs:173-221); the substep's
    // inputs are slot a's positions and velocities and its densities and pressures
    int32_t mover_felt(float dt, const Params& p, int a, int nid);

    // lift.rs:24-158: what the water does to each coupled body over dt, read as one smooth field
    // around it, from the committed positions and velocities (host copies in p, v)
    struct Lift {
        size_t owner;
        F3 impulse, angular;
        std::vector<uint32_t> near;  // the particles read, as places in the lift's P and V
    };
    // The region a body's lift reads (lift.rs:40-52): its probes placed by the pose (arm from the
    // centre, velocity), and their box grown by three kernel radii.
    void lift_region(const Coupled& known, const slf_body_pose& state, std::vector<std::pair<F3, F3>>& probes,
                     F3& low, F3& high) const;
    // P, V: the particles inside the bodies' regions (read_lift_water), in index order.
    std::vector<Lift> lifts(float dt, const slf_body_pose* poses, uint64_t npose, const std::vector<F3>& P,
                            const std::vector<F3>& V) const;
    // The particles inside any of the boxes, selected and compacted on the device in index order,
    // read back with their indexes: the lift reads these and not the whole state.
    DevBuf<uint32_t> lkeep, lat, lidx, ltiles;
    DevBuf<float> lpv;
    DevBuf<float3> lboxes;
    int32_t read_lift_water(const std::vector<float3>& boxes, std::vector<uint32_t>& index, std::vector<F3>& P,
                            std::vector<F3>& V);
    // the velocities of the particles read_lift_water read last, written back in the same order
    int32_t write_lift_velocities(const std::vector<F3>& V);

    // couple.rs:219-248 with the rigid world left to the caller
    int32_t step_with_bodies(float dt, const slf_body_pose* poses, uint64_t npose, slf_report* out,
                             std::vector<slf_body_push>& pushes);

    // ---- walls (src/fluid/boundary.rs) -------------------------------------------------------

    static int32_t check_box(const float* low, const float* high);

    void cells_in(const float* low, const float* high, int64_t out[3]) const;

    int32_t check_room(int64_t count) const;

    uint32_t add_wall_points(const std::vector<F3>& pts);

    int32_t add_box_container(const float* low, const float* high, uint32_t* out);

    int32_t add_wall(const float* low, const float* high, uint32_t* out);

    bool remove_boundary(uint32_t id);

    void update_bounds();

    static uint32_t fbits(float v);

    // settle_walls (boundary.rs:155-178): sort by cell, owner, position bits, index.
    void settle_walls();

    // The cell table of points sorted by cell (keys in order, m = keys.size()): dense over their
    // box while it holds at most 64 cells per occupied one plus 4096 (mod.rs:214-216), else the
    // occupied cells for search; uploaded into dstart / dkeys, described by g.
    int32_t grid_from_keys(const std::vector<Key3>& keys, GridDev& g, DevBuf<uint32_t>& dstart, DevBuf<int4>& dkeys);

    // Uploads the walls and their cell table: dense over the walls' box while it holds at most 64
    // cells per occupied one plus 4096 (mod.rs:214-216), else the occupied cells for search.
    int32_t upload_walls();

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
    static Status fresh_status();
    int32_t reset_status();

    // Box of cells and fastest speed of the committed state.
    int32_t refresh_stats();

    float fastest() const { float v; uint32_t b = h_status->vmax_bits; std::memcpy(&v, &b, 4); return v; }

    // ---- the spatial hash (update_neighbors, src/fluid/mod.rs:540-566) ------------------------

    // Sorts the committed state into slot `to` (pos/vel) and the other id slot, by (cell, id).
    // Needs the committed state's box in the status.  Commits nothing.
    int32_t sort_into(int to);

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
    int32_t plan_sort(SortPlan& sp, bool stable);

    // the planned sort's launches on stream `on`
    int32_t enqueue_sort(int to, const SortPlan& sp, cudaStream_t on);

    int32_t update_neighbors();

    int32_t compute_densities();

    // ---- substeps ----------------------------------------------------------------------------

    // one WCSPH substep (step.rs:144-224) from the committed state; commits on success
    int32_t wcsph_substep(float dt, uint32_t& held);

    // solve (dfsph.rs:222-275): Jacobi iterations until the average error is under tolerance.
    // Iterations are queued in batches; the device counts them and turns the launches after
    // the stopping check into no-ops, so the host waits once a batch instead of once an
    // iteration.  A batch is as long as the last solve of the same kind took.
    uint32_t expected_iterations[2] = {2, 2};
    int32_t solve(int which, const Params& p, int a, float4* v, int nid, uint32_t& iterations,
                  SolveRec rec = SolveRec{nullptr, nullptr});

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
    // Solve graphs: a checkpoint segment's replay keeps each DFSPH substep's lists in that
    // substep's record, so a segment of k substeps brings k list sets, each solved twice in up
    // to six slot arrangements (12 k graphs); room for a 22-substep segment's 264.
    static constexpr size_t kSolveGraphCache = 300;
    // A DFSPH segment kept in its records (kept_dfsph_substep) saves each substep's third sort
    // and density pass, but its solves meet new graph keys until every record has come round in
    // every slot arrangement: with graphs the backward keeps segments only on tapes of at least
    // this many (C5's 251 gain 0.8 ms a substep; 4 segments of 8 substeps lost 130 ms).
    static constexpr size_t kKeepMinSegments = 32;
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
    void drop_solve_graphs();
    template <class T> static void key_add(std::vector<uint8_t>& k, const T& v) {
        const uint8_t* b = reinterpret_cast<const uint8_t*>(&v);
        k.insert(k.end(), b, b + sizeof(T));
    }
    static void key_lists(std::vector<uint8_t>& k, const PairLists& l);
    std::vector<uint8_t> solve_key(int which, const Params& p, int a, float4* v, int nid, const PairLists& fl,
                                   const PairLists& wl, const SolveRec& rec);

    // records the solve's launches into a new graph on cap[0] (the loop body on cap[1])
    int32_t capture_solve(int which, const Params& p, int a, float4* v, int nid, const PairLists& fl,
                          const PairLists& wl, const SolveRec& rec, uint32_t& pre);

    int32_t solve_graph(int which, const Params& p, int a, float4* v, int nid, const PairLists& fl,
                        const PairLists& wl, const SolveRec& rec, uint32_t& iterations);

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

    bool whole_substeps() const;
    void drop_substep_graphs();
    std::vector<uint8_t> substep_key(const Params& p, int a, int b, int nid, const SortPlan& sp);

    // records the substep's launches into g.exec (the solve loops' bodies on cap[1])
    int32_t capture_substep(const Params& p, int a, int b, int nid, const SortPlan& sp, SubstepGraph& g);

    // Runs the planned substep as one graph launch when its graph is cached or recorded now;
    // ran = false leaves the substep to the eager launches.
    int32_t substep_graph(float dt, const Params& p, int a, int b, int nid, const SortPlan& sp, bool& ran);

    // After solves that ran as graphs (status read back): their iteration counts, their loop
    // kernels in the launch count, and the checks the batched path makes per solve (the lists'
    // room, the stop flag).  its[w] is set for each solve w that ran.
    int32_t finish_graph_solves(uint32_t its[2]);

    // The launches of a solve after its stopping check did nothing; their profile entries
    // go under "solver_idle" so the kernels' averages hold only launches that worked.
    void relabel_idle(size_t first, const std::vector<int>& kinds, uint32_t iterations);

    // a solve's records land here, max_iterations + 1 slots, before they are kept
    DevBuf<float> rec_rate;
    DevBuf<float4> rec_vel;

    // Records are sized for a quarter more iterations than any solve has recorded yet, so the
    // records a later tape reuses seldom grow: a new device allocation in the middle of a taped
    // run costs far more than the substep.
    uint32_t record_room = 0;
    int32_t keep_record(uint32_t its, DevBuf<float>& rates, DevBuf<float4>& vels);

    // one DFSPH substep (dfsph.rs:79-103) from the committed state; commits on success.  With
    // `rec`, the solves are recorded for the adjoint (the same batched launches, the slot of
    // each check taken from the device's iteration count).
    int32_t dfsph_substep(float dt, uint32_t& held, uint32_t& iterations, DfsphRecord* rec = nullptr);
    uint32_t last_iterations[2] = {0, 0};

    // step (step.rs:58-90), recorded when a tape is on
    int32_t step(float dt, slf_report* out);

    // ---- the adjoint ---------------------------------------------------------------------------

    int32_t tape_begin(uint32_t every);

    // gives the recorded substeps from the keep-th on back to the spares
    void drop_records(size_t keep);

    // a new substep record holding the committed state, for a tape with every == 0
    int32_t record_begin(float dt);

    // the tape's buffers (records, checkpoints, solver scratch) stay for the next tape
    int32_t tape_end();

    // the committed state becomes checkpoint number ckpt_sub.size(), before substep tape.count
    // a substep of a recorded step: the checkpoint due before it (every k-th substep), then its length
    int32_t tape_substep(float dt);
    int32_t checkpoint();

    // the committed state (positions, velocities, ids and, for cell-relative positions, cells) to
    // and from device buffers of n entries; c may be null for absolute positions
    // (w: warm starts' impulses of each particle, copied when warm starts are on)
    int32_t save_state(float4* p, float4* v, uint32_t* id, int4* c, float2* w = nullptr);

    int32_t load_state(const float4* p, const float4* v, const uint32_t* id, const int4* c,
                       const float2* w = nullptr);

    int32_t substep_retrying(float dt);

    // The sort and density pass of a DFSPH substep from the committed state, without the
    // solves: the lists, factors and densities the adjoint of a recorded substep reads.  The
    // sort's destinations go to sort_dest.  Commits nothing; returns the slots used.
    int32_t dfsph_replay(float dt, int& a, int& nid);

    // step_backward: reverse over the taped steps, one checkpoint segment at a time.
    int32_t step_backward(const float* dpos, const float* dvel, uint64_t k, float* dpos0, float* dvel0,
                          slf_param_grads* out);

    // The substep's sensitivities to its derived constants, taken back to the settings:
    // nu = min(viscosity c r, 0.05 r^2 / dt) (step.rs:254-259), nu_w = min(c r, 0.25 r^2 / dt)
    // (step.rs:282-283), B = rest c^2 / 7 (step.rs:149); the branch the substep took decides.
    void accumulate_param_grads(float dt, const double* g, slf_param_grads& pg, float sound = 0.0f,
                                bool raised = false) const;

    int32_t step_untaped(float dt, slf_report* out);

    // Keeps, in order, the particles inside the box (drain = 0) or outside it (drain = 1);
    // `removed` counts the others.
    int32_t keep_where(F3 low, F3 high, int drain, uint32_t& removed);

    // keep_in_domain (mod.rs:451-486)
    int32_t keep_in_domain(uint32_t& lost);

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
    int32_t add_flow(const float* low, const float* high, bool emitter, const float* velocity, uint32_t* out);

    // remove_flow (flow.rs:109-113)
    bool remove_flow(uint32_t id);

    // Rust's `f as i64`: saturating, NaN to 0
    static int64_t as_i64(float v);

    // run_flows (flow.rs:144-231): drains first, then emitters, each in the order they were
    // added.  An emitter whose lattice would hold more than 2^30 slots is refused (the reference
    // allocates one flag per slot, up to 4096^3).
    int32_t run_flows(uint32_t& emitted, uint32_t& drained);

    // ---- snapshots (src/fluid/save.rs) ---------------------------------------------------------

    // save_snapshot (save.rs:18-73): the SLFL version 3 bytes of the current state, particles in
    // their current order; no coupled bodies or terrains exist on this path.
    int32_t save_snapshot(std::vector<uint8_t>& out);

    // load_snapshot (save.rs:79-181) into a fresh world: untrusted bytes, checked in the
    // reference's order; the library's own settings fields come from `lib`.
    int32_t load_snapshot(const uint8_t* data, size_t size, const slf_settings& lib);

    // ---- read-outs -------------------------------------------------------------------------

    // packs xyz on the device and copies 12 bytes a particle straight into the caller's buffer
    int32_t read_vec(const DevBuf<float4>& b, float* out, uint64_t k);

    // the committed positions as xyz triples (cell-relative ones rebuilt in double, rounded once)
    int32_t read_positions(float* out, uint64_t k);

    int32_t write_vec(DevBuf<float4>& b, const float* in, uint64_t k);

    // Uploads the caller's state into a free slot, checking it on the device as it unpacks and
    // folding the box and speed the next step needs, then waits once: a state with a non finite
    // value is refused and the committed one stays.
    int32_t write_state(const float* p, const float* v, uint64_t k);

    // positions and velocities into the caller's buffers with one wait
    int32_t read_state(float* p, float* v, uint64_t k);

    template <class T> int32_t read_plain(const DevBuf<T>& b, T* out, uint64_t k) {
        if (k) {
            SLF_CUDA(cudaMemcpyAsync(out, b.p, k * sizeof(T), cudaMemcpyDeviceToHost, stream));
            SLF_CUDA(cudaStreamSynchronize(stream));
        }
        return SLF_OK;
    }

    int32_t lists(bool walls, uint32_t* start, uint64_t start_len, uint32_t* items, uint64_t cap, uint64_t* len);

    uint64_t state_hash_host(const std::vector<uint32_t>& id, const std::vector<float>& p,
                             const std::vector<float>& v) const;
};

}  // namespace slf
