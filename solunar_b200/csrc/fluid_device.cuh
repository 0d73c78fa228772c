// fluid_device.cuh -- device-side types and the per-pair arithmetic of the fluid step.
//
// Kernels in this library are compiled with -fmad=false and IEEE division and square root, so
// that `a * b + c` rounds twice and every expression below rounds exactly as the reference's
// scalar f32 code (src/fluid/mod.rs, step.rs, dfsph.rs) does.  The formulas keep the
// reference's evaluation order; each cites the line it follows.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace slf {

constexpr int kBlock = 256;           // threads per block of the per-particle kernels
constexpr uint32_t kNoCell = 0xFFFFFFFFu;

// ---- world constants, derived once from the settings on the host (in f32, reference order) --
struct Params {
    float spacing;
    float radius;        // spacing * support (mod.rs:120-122)
    float reach;         // radius.powi(2) (mod.rs:568)
    float scale;         // 21 / (2 pi r^3) (mod.rs:136)
    float mass;          // rest_mass (mod.rs:694-709)
    float rest;          // rest_density
    float rest_sq;       // rest * rest (step.rs:198)
    float stiffness;     // rest * c^2 / 7 (step.rs:149)
    float soften;        // 0.01 * r * r (step.rs:165)
    float3 gravity;
    int has_bounds;      // a container exists (boundary.rs:240-247)
    float3 low, high;    // union of the containers
    float3 low_in, high_in;  // low + spacing/2, high - spacing/2 (step.rs:308-312)
    uint32_t n;          // particles
    int solver;          // 0 WCSPH, 1 DFSPH
    float div_tol, den_tol;
    uint32_t min_iter, max_iter;
    // reciprocal constants of the FAST arithmetic
    float inv_radius;      // 1 / r
    float grad_scale;      // scale * (-20) / r^2: slope(d) / d = grad_scale * (1 - d / r)^3
    float inv_rest;        // 1 / rest_density
    float inv_rest_sq;     // 1 / rest_density^2
    float settles;         // |gravity| spacing: the speed under which water settles on a body (couple.rs:390)
};

// Per-substep constants, in device memory so a captured substep reads the current ones.
struct StepConsts {
    float dt;
    float viscosity;       // viscosity(dt) (step.rs:254-259)
    float wall_viscosity;  // min(c r, 0.25 r^2 / dt) (step.rs:282-283)
    float dt_sq;           // dt * dt (dfsph.rs:246)
    float mover_damping;   // min(1 c r, 0.25 r r / dt), the body points' damping (step.rs:163-164)
};

// Written by the kernels, read back by the host after each substep.
struct Status {
    uint32_t nonfinite;    // advance found a non finite particle (step.rs:333-335)
    uint32_t held;         // held_back of the substep (step.rs:314-316)
    uint32_t vmax_bits;    // max |v| of the advanced state, f32 bits (non-negative)
    uint32_t maxcomp_bits; // max(0, rho / rest - 1), f32 bits
    int32_t cell_lo[3];    // bounding box of the advanced particles' cells
    int32_t cell_hi[3];
    uint32_t settled;      // the last solver check stopped the loop
    uint32_t loaded;       // particles with error > 0 in the last check (dfsph.rs:266)
    double average;        // last average error (dfsph.rs:267)
    uint32_t processed;    // particles a neighbour pass visited (dispatch completeness)
    uint32_t ticket;       // block counter of the last-block reduction
    uint32_t list_max;     // longest neighbour list the last density pass found
    uint32_t iterations;   // pushes of the running solve so far (dfsph.rs:236, 273)
    uint32_t solved[2];    // pushes of the last divergence (0) and density (1) solve, set when it stops
    uint32_t bodies;       // loop bodies a solve run as a CUDA graph has started
    uint32_t overrun;      // such a solve passed max_iterations + 1 bodies and was stopped
};

// What a solver check records for the adjoint (both null: nothing): at slot it = the solve's
// iteration count when the check runs, rate[it * n + i] = the density rate of particle i and
// vel[it * n + i] = the velocity it read.  The device stops a solve at max_iterations, so
// max_iterations + 1 slots always suffice.
struct SolveRec {
    float* rate;
    float4* vel;
};

// Neighbour lists of one substep, built by the density pass in the reference's list order
// (mod.rs:570-606) and read by every later pass of the substep.  An entry is 8 bytes: the
// neighbour's index and its kernel gradient factor g = slope(d) / d (0 at d = 0), kept because
// positions do not move within a substep (the reference keeps the whole gradient per pair for
// the same reason, dfsph.rs:24-41); gradient = offset * g rounds as Kernel::gradient does
// (mod.rs:158-164).  Layout: warp tiles, entry k of row s at ((s / 32) * cap + k) * 32 + s % 32,
// so a warp reading slot k of its 32 rows reads 256 contiguous bytes and each warp's lists are
// one contiguous block.  Rows follow the walk order: thread s of a list pass walks particle
// order[s] (identity when order is null) and its list is row s.  The order visits the cells in 2 x 2-column bricks
// (the world builds it after each sort), so a block's 256 particles span about 2 x 2 x 8 cells and
// their neighbourhoods overlap in the L1; particle arrays stay in the reference's sorted order.
//
// EXACT DFSPH also keeps each pair's whole gradient, as the reference's gradient cache does
// (dfsph.rs:24-41): gv, at the same slots, holds {offset.x * g, offset.y * g, offset.z * g,
// index bits} (walls: index 0).  The density pass writes it when gv is set; the solver check then
// streams it and gathers only the neighbour's velocity, where from (index, g) it would gather the
// position as well.  The products are the ones every pass forms, so the bits are the same.
struct PairLists {
    uint32_t cap;          // slots per row
    uint2* e;              // entries {index, g bits}
    uint32_t* count;       // neighbours found per row; above cap the lists are incomplete
    const uint32_t* order; // particle of each row (null: row = particle)
    float4* gv;            // gradient entries (null: not kept)

    __host__ __device__ static size_t slots_for(uint32_t n, uint32_t cap) {
        return size_t((n + 31u) / 32u) * cap * 32u;
    }
    __host__ __device__ size_t at(uint32_t row, uint32_t k) const {
        return (size_t(row >> 5) * cap + k) * 32u + (row & 31u);
    }
#ifdef __CUDACC__
    __device__ __forceinline__ uint32_t particle(uint32_t row) const { return order ? __ldg(&order[row]) : row; }
#endif
};

// Terrain regions (src/fluid/terrain.rs): signed distances at nodes `step` apart from `low`, index
// (y * nz + z) * nx + x, `offset` into the shared distance array; and the ground sites, the
// water's lattice within the kernel around a particle with the density each site adds.
struct TerrainRegion {
    float lx, ly, lz;
    float step;
    uint32_t nx, ny, nz;
    uint32_t pad;
    unsigned long long offset;
};
struct TerrainDev {
    uint32_t regions;              // 0: no terrain (every term below is skipped)
    uint32_t sites;
    const TerrainRegion* region;
    const float* dist;
    const float4* site;            // offset xyz, density weight
    const float* far;              // |offset|
    const float* damping;          // kGroundSamples weights from `low` in steps of `step`
    float spacing, reach, low, step;
};
constexpr int kGroundSamples = 256;

// Slots of the adjoint's FP64 parameter-gradient accumulators.
enum GradSlot { kGradViscosity = 0, kGradWallViscosity = 1, kGradStiffness = 2, kGradGravity = 3, kGradSlots = 6 };

// ---- cell tables ----------------------------------------------------------------------------
// Dense: a start offset for every cell of a box, x-major like the reference's dense table
// (mod.rs:218-223): range of cell c = [start[c], start[c + 1]).  Sorted: the occupied cells'
// keys in key order with their starts, searched like the reference's fallback (mod.rs:231).
struct GridDev {
    int mode;              // 0 empty, 1 dense, 2 sorted
    int lx, ly, lz;        // dense: lowest key
    int sx, sy, sz;        // dense: cells per axis
    uint32_t cells;        // sorted: occupied cells
    const uint32_t* start; // dense: volume + 1; sorted: cells + 1
    const int4* keys;      // sorted: key of each occupied cell

#ifdef __CUDACC__
    __device__ __forceinline__ bool range(long long cx, long long cy, long long cz, uint32_t& b,
                                          uint32_t& e) const {
        if (mode == 1) {
            long long x = cx - lx, y = cy - ly, z = cz - lz;
            if (x < 0 || x >= sx || y < 0 || y >= sy || z < 0 || z >= sz) return false;
            long long c = (x * sy + y) * sz + z;
            b = start[c];
            e = start[c + 1];
            return e > b;
        }
        if (mode == 2) {
            if (cx > 2147483647LL || cx < -2147483648LL || cy > 2147483647LL || cy < -2147483648LL ||
                cz > 2147483647LL || cz < -2147483648LL)
                return false;
            uint32_t lo = 0, hi = cells;
            while (lo < hi) {
                uint32_t mid = (lo + hi) >> 1;
                int4 k = keys[mid];
                bool less = k.x < cx || (k.x == cx && (k.y < cy || (k.y == cy && k.z < cz)));
                if (less) lo = mid + 1;
                else hi = mid;
            }
            if (lo == cells) return false;
            int4 k = keys[lo];
            if (k.x != cx || k.y != cy || k.z != cz) return false;
            b = start[lo];
            e = start[lo + 1];
            return true;
        }
        return false;
    }
#endif
};

// The points of the coupled bodies for the running substep (couple.rs:35-47), sorted by
// (cell, owner, place) with their cell table: positions with the owner's index in w (as bits),
// velocities.  count = 0: no bodies, every term is skipped.
struct MoverDev {
    uint32_t count;
    GridDev grid;
    const float4* pos;
    const float4* vel;
};

#ifdef __CUDACC__

// Neighbour lists (a few hundred MB at a million particles, more than the L2) are written once
// a substep and streamed once by each later pass: their loads are evict-first, so they do not
// push the particle arrays the passes gather from out of the L2.
#ifndef SLF_LIST_LOAD
#define SLF_LIST_LOAD __ldcs
#endif

// ---- reference arithmetic (mod.rs:125-165, 526-533) ------------------------------------------

__device__ __forceinline__ float pow3(float x) { return x * (x * x); }
__device__ __forceinline__ float pow4(float x) { float s = x * x; return s * s; }
__device__ __forceinline__ float pow7(float x) { float s = x * x; float q = s * s; return (x * s) * q; }

// x*x' + y*y' + z*z', left to right, each operation rounded on its own whatever the compiler's
// contraction setting: the neighbour test and the cell keys depend on these bits.
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// Kernel::value (mod.rs:140-146)
__device__ __forceinline__ float kernel_value(const Params& p, float distance) {
    float q = distance / p.radius;
    if (q >= 1.0f) return 0.0f;
    return p.scale * pow4(1.0f - q) * (1.0f + 4.0f * q);
}

// Kernel::slope (mod.rs:149-155)
__device__ __forceinline__ float kernel_slope(const Params& p, float distance) {
    float q = distance / p.radius;
    if (q >= 1.0f) return 0.0f;
    return p.scale * -20.0f * q * pow3(1.0f - q) / p.radius;
}

// Kernel::gradient (mod.rs:158-164): the factor g with gradient = offset * g.
__device__ __forceinline__ float kernel_gradient_factor(const Params& p, float ox, float oy, float oz) {
    float distance = sqrtf(dot3(ox, oy, oz, ox, oy, oz));
    if (distance <= 0.0f) return 0.0f;
    return kernel_slope(p, distance) / distance;
}

// cell_of (mod.rs:526-533): floor(p / r) per axis, `as i32` (PTX float-to-int conversions
// saturate and map NaN to zero, as Rust's does).
__device__ __forceinline__ int3 cell_of(const Params& p, float x, float y, float z) {
    return make_int3(__float2int_rz(floorf(__fdiv_rn(x, p.radius))), __float2int_rz(floorf(__fdiv_rn(y, p.radius))),
                     __float2int_rz(floorf(__fdiv_rn(z, p.radius))));
}

// ---- terrain fields (src/fluid/terrain.rs) ---------------------------------------------------
// Every operation is rounded on its own through the intrinsics, so the EXACT forward and the
// adjoint (compiled with contraction on) sample the same bits and take the same branches.

__device__ __forceinline__ float lerp_rn(float a, float b, float u) { return __fadd_rn(a, __fmul_rn(__fsub_rn(b, a), u)); }

// The corners of the field cell holding a point, and the point's place in it.
struct TerrainCell {
    float a00, b00, a10, b10, a01, b01, a11, b11;  // a: x low, b: x high; digits: y, z
    float fx, fy, fz;
};

// The cell of TerrainField::read (terrain.rs:100-136); false outside the region.
__device__ __forceinline__ bool terrain_cell(const TerrainDev& T, const TerrainRegion& t, float px, float py,
                                             float pz, TerrainCell& c) {
    float lx = __fdiv_rn(__fsub_rn(px, t.lx), t.step), ly = __fdiv_rn(__fsub_rn(py, t.ly), t.step),
          lz = __fdiv_rn(__fsub_rn(pz, t.lz), t.step);
    if (!(lx >= 0.0f && lx <= float(t.nx - 1) && ly >= 0.0f && ly <= float(t.ny - 1) && lz >= 0.0f &&
          lz <= float(t.nz - 1)))
        return false;
    uint32_t x = min(uint32_t(floorf(lx)), t.nx - 2), y = min(uint32_t(floorf(ly)), t.ny - 2),
             z = min(uint32_t(floorf(lz)), t.nz - 2);
    c.fx = __fsub_rn(lx, float(x));
    c.fy = __fsub_rn(ly, float(y));
    c.fz = __fsub_rn(lz, float(z));
    const float* d = T.dist + t.offset;
    auto corner = [&](uint32_t dx, uint32_t dy, uint32_t dz) {
        return __ldg(&d[(size_t(y + dy) * t.nz + (z + dz)) * t.nx + (x + dx)]);
    };
    c.a00 = corner(0, 0, 0), c.b00 = corner(1, 0, 0), c.a10 = corner(0, 1, 0), c.b10 = corner(1, 1, 0);
    c.a01 = corner(0, 0, 1), c.b01 = corner(1, 0, 1), c.a11 = corner(0, 1, 1), c.b11 = corner(1, 1, 1);
    return true;
}

// The trilinear distance in a cell and its change per axis (terrain.rs:100-136).
__device__ __forceinline__ void terrain_values(const TerrainCell& c, float step, float& value, float3& change) {
    float v00 = lerp_rn(c.a00, c.b00, c.fx), g00 = __fsub_rn(c.b00, c.a00);
    float v10 = lerp_rn(c.a10, c.b10, c.fx), g10 = __fsub_rn(c.b10, c.a10);
    float v01 = lerp_rn(c.a01, c.b01, c.fx), g01 = __fsub_rn(c.b01, c.a01);
    float v11 = lerp_rn(c.a11, c.b11, c.fx), g11 = __fsub_rn(c.b11, c.a11);
    float v0 = lerp_rn(v00, v10, c.fy), v1 = lerp_rn(v01, v11, c.fy);
    value = lerp_rn(v0, v1, c.fz);
    change = make_float3(__fdiv_rn(lerp_rn(lerp_rn(g00, g10, c.fy), lerp_rn(g01, g11, c.fy), c.fz), step),
                         __fdiv_rn(lerp_rn(__fsub_rn(v10, v00), __fsub_rn(v11, v01), c.fz), step),
                         __fdiv_rn(__fsub_rn(v1, v0), step));
}

// TerrainField::read (terrain.rs:100-136): the trilinear distance at a point and its change per
// axis; false outside the region.
__device__ __forceinline__ bool terrain_read(const TerrainDev& T, const TerrainRegion& t, float px, float py,
                                             float pz, float& value, float3& change) {
    TerrainCell c;
    if (!terrain_cell(T, t, px, py, pz, c)) return false;
    terrain_values(c, t.step, value, change);
    return true;
}

// normalize_or(Y) dividing by the length
__device__ __forceinline__ float3 normalize_or_up(float3 c) {
    float len = __fsqrt_rn(dot3(c.x, c.y, c.z, c.x, c.y, c.z));
    if (isfinite(len) && len > 0.0f) return make_float3(__fdiv_rn(c.x, len), __fdiv_rn(c.y, len), __fdiv_rn(c.z, len));
    return make_float3(0.0f, 1.0f, 0.0f);
}

// TerrainField::sample (terrain.rs:139-142)
__device__ __forceinline__ bool terrain_sample(const TerrainDev& T, const TerrainRegion& t, float px, float py,
                                               float pz, float& distance, float3& normal) {
    float3 change;
    if (!terrain_read(T, t, px, py, pz, distance, change)) return false;
    normal = normalize_or_up(change);
    return true;
}

// One region of terrain_contact (terrain.rs:314-333): a particle at (x, y, z) nearer the
// region's surface than `rest` goes back there and its velocity into the surface is removed.
// Returns whether it was nearer; under: whether it was beneath the surface.
__device__ __forceinline__ bool contact_region(const TerrainDev& T, const TerrainRegion& t, float rest, float& x,
                                               float& y, float& z, float4& v, bool& under) {
    float distance;
    float3 gn;
    if (!terrain_sample(T, t, x, y, z, distance, gn)) return false;
    if (!(distance < rest)) return false;
    under = under || distance < 0.0f;
    float lift = __fsub_rn(rest, distance);
    x = __fadd_rn(x, __fmul_rn(gn.x, lift));
    y = __fadd_rn(y, __fmul_rn(gn.y, lift));
    z = __fadd_rn(z, __fmul_rn(gn.z, lift));
    float into = dot3(v.x, v.y, v.z, gn.x, gn.y, gn.z);
    if (into < 0.0f) {
        v.x = __fsub_rn(v.x, __fmul_rn(gn.x, into));
        v.y = __fsub_rn(v.y, __fmul_rn(gn.y, into));
        v.z = __fsub_rn(v.z, __fmul_rn(gn.z, into));
    }
    return true;
}

// GroundSites::damping (terrain.rs:241-249); slope (optional): its derivative in the distance
__device__ __forceinline__ float ground_damping(const TerrainDev& T, float distance, float* slope = nullptr) {
    float at = __fdiv_rn(__fsub_rn(fmaxf(distance, T.low), T.low), T.step);
    uint32_t below = uint32_t(floorf(at));
    if (slope) *slope = 0.0f;
    if (below + 1 >= uint32_t(kGroundSamples)) return 0.0f;
    float part = __fsub_rn(at, float(below));
    float d0 = __ldg(&T.damping[below]), d1 = __ldg(&T.damping[below + 1]);
    if (slope && distance > T.low) *slope = (d1 - d0) / T.step;
    return __fadd_rn(d0, __fmul_rn(__fsub_rn(d1, d0), part));
}

// The candidates of one cell, points [b, e), two gathers in flight at a time; f(j, q) for each
// point within reach, in array order.
template <class F>
__device__ __forceinline__ void each_in_cell(const Params& p, const float4* __restrict__ pts, uint32_t b,
                                             uint32_t e, float ax, float ay, float az, F&& f) {
    uint32_t j = b;
#pragma unroll 1
    for (; j + 1 < e; j += 2) {
        float4 q0 = __ldg(&pts[j]), q1 = __ldg(&pts[j + 1]);
        float ox = q0.x - ax, oy = q0.y - ay, oz = q0.z - az;
        if (dot3(ox, oy, oz, ox, oy, oz) < p.reach) f(j, q0);
        ox = q1.x - ax, oy = q1.y - ay, oz = q1.z - az;
        if (dot3(ox, oy, oz, ox, oy, oz) < p.reach) f(j + 1, q1);
    }
    if (j < e) {
        float4 q = __ldg(&pts[j]);
        float ox = q.x - ax, oy = q.y - ay, oz = q.z - az;
        if (dot3(ox, oy, oz, ox, oy, oz) < p.reach) f(j, q);
    }
}

// Visit the points of `g` within reach of `at` in the reference's list order: the 27 cells
// dz outer, dy, dx inner (mod.rs:250-261), each cell's points in array order, kept when
// |p - at|^2 < reach strictly (mod.rs:264-277).
template <class F>
__device__ __forceinline__ void each_near(const Params& p, const GridDev& g, const float4* __restrict__ pts,
                                          int3 cell, float ax, float ay, float az, F&& f) {
    // the offsets below are single subtractions and the test uses dot3: exact under any flags
    if (g.mode == 0) return;
    if (g.mode == 1) {
        // dense table (under 2^31 cells): the cell's place in it once, in 64 bits as cells near
        // the i32 limits overflow, each neighbour's index in 32 bits once it is known inside
        const long long bx = (long long)cell.x - g.lx, by = (long long)cell.y - g.ly, bz = (long long)cell.z - g.lz;
#pragma unroll 1
        for (int dz = -1; dz <= 1; ++dz) {
            long long z = bz + dz;
            if (z < 0 || z >= g.sz) continue;
#pragma unroll 1
            for (int dy = -1; dy <= 1; ++dy) {
                long long y = by + dy;
                if (y < 0 || y >= g.sy) continue;
                uint32_t yz = uint32_t(y) * uint32_t(g.sz) + uint32_t(z);
#pragma unroll 1
                for (int dx = -1; dx <= 1; ++dx) {
                    long long x = bx + dx;
                    if (x < 0 || x >= g.sx) continue;
                    uint32_t c = uint32_t(x) * (uint32_t(g.sy) * uint32_t(g.sz)) + yz;
                    uint32_t b = __ldg(&g.start[c]), e = __ldg(&g.start[c + 1]);
                    if (e > b) each_in_cell(p, pts, b, e, ax, ay, az, f);
                }
            }
        }
        return;
    }
#pragma unroll 1
    for (int dz = -1; dz <= 1; ++dz) {
#pragma unroll 1
        for (int dy = -1; dy <= 1; ++dy) {
#pragma unroll 1
            for (int dx = -1; dx <= 1; ++dx) {
                uint32_t b, e;
                if (!g.range((long long)cell.x + dx, (long long)cell.y + dy, (long long)cell.z + dz, b, e))
                    continue;
#pragma unroll 1
                for (uint32_t j = b; j < e; ++j) {
                    float4 q = __ldg(&pts[j]);
                    float ox = q.x - ax, oy = q.y - ay, oz = q.z - az;
                    if (dot3(ox, oy, oz, ox, oy, oz) < p.reach) f(j, q);
                }
            }
        }
    }
}

// f32 bits for atomicMax on non-negative floats.
__device__ __forceinline__ void atomic_max_nonneg(uint32_t* addr, float v) {
    if (v > 0.0f) atomicMax(addr, __float_as_uint(v));
}

#endif  // __CUDACC__

}  // namespace slf
