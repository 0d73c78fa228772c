// kernels_fast.cu -- the FAST arithmetic variants of the pair passes (SLF_ARITHMETIC_FAST).
//
// Same physics, same neighbours in the same order, same per-particle sums: only the rounding
// differs.  This file is compiled with contraction on, and the kernel is evaluated from
// reciprocal constants: with q = d / r, the gradient factor slope(d) / d of Kernel::gradient
// (src/fluid/mod.rs:149-164) is scale * (-20) * (1 - q)^3 / r^2, so a pair needs one reciprocal
// square root and a few fused multiply-adds instead of a square root and three divisions.  The
// neighbour lists hold indexes only (4 bytes an entry): each pass recomputes the factor from the
// positions, which do not move within a substep.  Cell keys and the neighbour test stay exact
// (fluid_device.cuh), so cell order and neighbour sets still match the reference bit for bit.
//
// Cell-relative positions (SLF_POSITIONS_CELL_RELATIVE, template flag REL): a particle's position
// is an f32 offset in [0, r) from the corner of its cell, its cell an integer triple beside it, and
// walls are stored the same way.  A pair's offset x_i - x_j = (o_i - o_j) - (c_j - c_i) r is then
// formed from small numbers; the cell step c_j - c_i (each -1, 0 or 1) rides in the top six bits
// of the list entry, so no pass gathers cells.
#include <cfloat>
#include <climits>

#include <atomic>

#include "fluid_device.cuh"
#include "launch.h"
#include "reduce.cuh"

namespace slf {

// List entries: the neighbour's index in the low 26 bits, the cell step to it (dx, dy, dz, each
// stored + 1) in the top 6.
constexpr uint32_t kIndexMask = (1u << 26) - 1u;
__device__ __forceinline__ uint32_t encode_entry(uint32_t j, int dx, int dy, int dz) {
    return j | (uint32_t((dx + 1) | ((dy + 1) << 2) | ((dz + 1) << 4)) << 26);
}

// x_i - x_j from particle i's stored position a and neighbour q's, given the entry e
template <bool REL>
__device__ __forceinline__ float3 pair_offset(const Params& p, float4 a, float4 q, uint32_t e) {
    if (!REL) return make_float3(a.x - q.x, a.y - q.y, a.z - q.z);
    float dx = float(int((e >> 26) & 3u) - 1), dy = float(int((e >> 28) & 3u) - 1),
          dz = float(int((e >> 30) & 3u) - 1);
    return make_float3(fmaf(-dx, p.radius, a.x - q.x), fmaf(-dy, p.radius, a.y - q.y),
                       fmaf(-dz, p.radius, a.z - q.z));
}

// Index-only lists in the warp-tiled layout of PairLists, 4 bytes an entry.
struct IndexLists {
    uint32_t cap;
    uint32_t* idx;
    uint32_t* count;
    __device__ size_t at(uint32_t i, uint32_t k) const { return (size_t(i >> 5) * cap + k) * 32u + (i & 31u); }
};

__device__ __forceinline__ IndexLists index_lists(const PairLists& l) {
    return IndexLists{l.cap, reinterpret_cast<uint32_t*>(l.e), l.count};
}

// q = d / r and the gradient factor slope(d) / d; zero at d = 0 as Kernel::gradient is.
__device__ __forceinline__ float fast_factor(const Params& p, float l2) {
    if (l2 <= 0.0f) return 0.0f;
    float d = l2 * rsqrtf(l2);
    float om = fmaxf(1.0f - d * p.inv_radius, 0.0f);
    return p.grad_scale * (om * om * om);
}

// Kernel::value (mod.rs:140-146) from the squared distance.
__device__ __forceinline__ float fast_value(const Params& p, float l2) {
    float d = l2 > 0.0f ? l2 * rsqrtf(l2) : 0.0f;
    float q = d * p.inv_radius;
    float om = fmaxf(1.0f - q, 0.0f);
    float om2 = om * om;
    return p.scale * (om2 * om2) * fmaf(4.0f, q, 1.0f);
}

__device__ __forceinline__ float fl2(float x, float y, float z) { return fmaf(x, x, fmaf(y, y, z * z)); }

// Where a walk finds its neighbours (the global arrays, read through the L1).
struct FromGlobalF {
    const float4* __restrict__ p;
    const float4* __restrict__ v;
    __device__ __forceinline__ void get(uint32_t e, float4& q) const { q = __ldg(&p[e & kIndexMask]); }
    __device__ __forceinline__ void get(uint32_t e, float4& q, float4& w) const {
        q = __ldg(&p[e & kIndexMask]);
        w = __ldg(&v[e & kIndexMask]);
    }
};

// f(entry, q) for each listed neighbour, q its stored position: four entries' gathers issued
// together, and the next four entries requested before these are used (past the end of the
// list the last entry is loaded again, a valid address, and not used)
template <class Src, class F>
__device__ __forceinline__ void each_index_from(const IndexLists& l, uint32_t i, const Src& src, F&& f) {
    uint32_t n = l.count[i];
    if (n > l.cap) n = l.cap;
    if (n == 0) return;
    const uint32_t* __restrict__ base = l.idx + l.at(i, 0);
    uint32_t e[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) e[u] = SLF_LIST_LOAD(base + size_t(u < (int)n ? u : n - 1) * 32u);
    for (uint32_t k = 0; k < n; k += 4) {
        float4 q[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) src.get(e[u], q[u]);
        uint32_t next[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            uint32_t kk = k + 4 + u;
            next[u] = SLF_LIST_LOAD(base + size_t(kk < n ? kk : n - 1) * 32u);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k + u < n) f(e[u], q[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u) e[u] = next[u];
    }
}

template <class F>
__device__ __forceinline__ void each_index(const IndexLists& l, uint32_t i, const float4* __restrict__ pts, F&& f) {
    each_index_from(l, i, FromGlobalF{pts, nullptr}, f);
}

template <class Src, class F>
__device__ __forceinline__ void each_index2_from(const IndexLists& l, uint32_t i, const Src& src, F&& f) {
    uint32_t n = l.count[i];
    if (n > l.cap) n = l.cap;
    if (n == 0) return;
    const uint32_t* __restrict__ base = l.idx + l.at(i, 0);
    uint32_t e[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) e[u] = SLF_LIST_LOAD(base + size_t(u < (int)n ? u : n - 1) * 32u);
    for (uint32_t k = 0; k < n; k += 4) {
        float4 q[4], w[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) src.get(e[u], q[u], w[u]);
        uint32_t next[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            uint32_t kk = k + 4 + u;
            next[u] = SLF_LIST_LOAD(base + size_t(kk < n ? kk : n - 1) * 32u);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k + u < n) f(e[u], q[u], w[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u) e[u] = next[u];
    }
}

template <class F>
__device__ __forceinline__ void each_index2(const IndexLists& l, uint32_t i, const float4* __restrict__ pts,
                                            const float4* __restrict__ more, F&& f) {
    each_index2_from(l, i, FromGlobalF{pts, more}, f);
}

// The candidates of each_near (fluid_device.cuh) in cell-relative form: the 27 cells around
// `cell` in the same order, a candidate kept when |x_j - x_i|^2 < reach, x_j - x_i formed from
// the offsets and the cell step.  f(j, q, dx, dy, dz, rx, ry, rz) with r = x_i - x_j.
template <class F>
__device__ __forceinline__ void each_near_rel(const Params& p, const GridDev& g, const float4* __restrict__ pts,
                                              int3 cell, float4 a, F&& f) {
    if (g.mode == 0) return;
    if (g.mode == 1) {
        // dense table: as each_near's walk, the cell's place once, neighbours' indices in 32 bits
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
                    float sx = float(dx) * p.radius, sy = float(dy) * p.radius, sz = float(dz) * p.radius;
                    uint32_t j = b;
#pragma unroll 1
                    for (; j + 1 < e; j += 2) {
                        float4 q0 = __ldg(&pts[j]), q1 = __ldg(&pts[j + 1]);
                        float rx = (a.x - q0.x) - sx, ry = (a.y - q0.y) - sy, rz = (a.z - q0.z) - sz;
                        if (dot3(rx, ry, rz, rx, ry, rz) < p.reach) f(j, q0, dx, dy, dz, rx, ry, rz);
                        rx = (a.x - q1.x) - sx, ry = (a.y - q1.y) - sy, rz = (a.z - q1.z) - sz;
                        if (dot3(rx, ry, rz, rx, ry, rz) < p.reach) f(j + 1, q1, dx, dy, dz, rx, ry, rz);
                    }
                    if (j < e) {
                        float4 q = __ldg(&pts[j]);
                        float rx = (a.x - q.x) - sx, ry = (a.y - q.y) - sy, rz = (a.z - q.z) - sz;
                        if (dot3(rx, ry, rz, rx, ry, rz) < p.reach) f(j, q, dx, dy, dz, rx, ry, rz);
                    }
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
                if (!g.range((long long)cell.x + dx, (long long)cell.y + dy, (long long)cell.z + dz, b, e)) continue;
                float sx = float(dx) * p.radius, sy = float(dy) * p.radius, sz = float(dz) * p.radius;
#pragma unroll 1
                for (uint32_t j = b; j < e; ++j) {
                    float4 q = __ldg(&pts[j]);
                    float rx = (a.x - q.x) - sx, ry = (a.y - q.y) - sy, rz = (a.z - q.z) - sz;
                    if (dot3(rx, ry, rz, rx, ry, rz) < p.reach) f(j, q, dx, dy, dz, rx, ry, rz);
                }
            }
        }
    }
}

// ---- densities and lists (mod.rs:621-675; step.rs:147-172; dfsph.rs:108-163) ---------------

template <int SOLVER, bool REL>
__global__ void __launch_bounds__(kBlock) k_density_fast(Params p, GridDev fg, GridDev wg,
                                                         const float4* __restrict__ pos,
                                                         const int4* __restrict__ cells,
                                                         const float4* __restrict__ walls, PairLists fpl,
                                                         PairLists wpl, float* __restrict__ rho,
                                                         float* __restrict__ press, float* __restrict__ scaled,
                                                         float* __restrict__ alpha, Status* st) {
    IndexLists fl = index_lists(fpl), wl = index_lists(wpl);
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = row < p.n ? fpl.particle(row) : row;  // row of the walk order, its particle
    bool valid = i < p.n;
    uint32_t compressed = 0, longest = 0;
    if (valid) {
        float4 a = pos[i];
        int3 cell;
        if (REL) {
            int4 c4 = cells[i];
            cell = make_int3(c4.x, c4.y, c4.z);
        } else {
            cell = cell_of(p, a.x, a.y, a.z);
        }
        float sum = 0.0f, wsum = 0.0f;
        float sx = 0.0f, sy = 0.0f, sz = 0.0f, squares = 0.0f;
        uint32_t nf = 0, nw = 0;
        auto fluid = [&](uint32_t j, int dx, int dy, int dz, float rx, float ry, float rz) {
            float l2 = fl2(rx, ry, rz);
            sum += fast_value(p, l2);
            if (nf < fl.cap) fl.idx[fl.at(row, nf)] = encode_entry(j, dx, dy, dz);
            ++nf;
            if (SOLVER == 1) {
                float g = fast_factor(p, l2) * p.mass;
                float px = rx * g, py = ry * g, pz = rz * g;
                sx += px;
                sy += py;
                sz += pz;
                squares = fmaf(px, px, fmaf(py, py, fmaf(pz, pz, squares)));
            }
        };
        auto wall = [&](uint32_t j, int dx, int dy, int dz, float rx, float ry, float rz) {
            float l2 = fl2(rx, ry, rz);
            wsum += fast_value(p, l2);
            if (nw < wl.cap) wl.idx[wl.at(row, nw)] = encode_entry(j, dx, dy, dz);
            ++nw;
            if (SOLVER == 1) {
                float g = fast_factor(p, l2) * p.mass;
                sx = fmaf(rx, g, sx);
                sy = fmaf(ry, g, sy);
                sz = fmaf(rz, g, sz);
            }
        };
        if (REL) {
            each_near_rel(p, fg, pos, cell, a, [&](uint32_t j, float4, int dx, int dy, int dz, float rx, float ry,
                                                   float rz) { fluid(j, dx, dy, dz, rx, ry, rz); });
            each_near_rel(p, wg, walls, cell, a, [&](uint32_t j, float4, int dx, int dy, int dz, float rx, float ry,
                                                     float rz) { wall(j, dx, dy, dz, rx, ry, rz); });
        } else {
            each_near(p, fg, pos, cell, a.x, a.y, a.z,
                      [&](uint32_t j, float4 q) { fluid(j, 0, 0, 0, a.x - q.x, a.y - q.y, a.z - q.z); });
            each_near(p, wg, walls, cell, a.x, a.y, a.z,
                      [&](uint32_t j, float4 q) { wall(j, 0, 0, 0, a.x - q.x, a.y - q.y, a.z - q.z); });
        }
        fl.count[row] = nf;
        wl.count[row] = nw;
        longest = nf > nw ? nf : nw;
        float density = p.mass * (sum + wsum);
        rho[i] = density;
        if (SOLVER == 0) {
            float ratio = fminf(density * p.inv_rest, 1.1f);
            float r2 = ratio * ratio, r4 = r2 * r2;
            float pressure = fmaxf(p.stiffness * (ratio * r2 * r4 - 1.0f), 0.0f);
            press[i] = pressure;
            scaled[i] = pressure / (density * density);
        } else {
            float total = fl2(sx, sy, sz) + squares;
            alpha[i] = total > 0.0f ? 1.0f / total : 0.0f;
        }
        float c = density * p.inv_rest - 1.0f;
        if (c > 0.0f) compressed = __float_as_uint(c);
    }
    compressed = block_reduce(compressed, MaxU(), 0u);
    longest = block_reduce(longest, MaxU(), 0u);
    if (threadIdx.x == 0) {
        if (compressed) atomicMax(&st->maxcomp_bits, compressed);
        if (longest) atomicMax(&st->list_max, longest);
    }
}

// ---- wall viscosity (step.rs:262-301) --------------------------------------------------------

template <bool REL>
__device__ __forceinline__ float3 wall_viscous_fast(const Params& p, float wall_visc, const IndexLists& wl,
                                                    const float4* __restrict__ walls, uint32_t row, float4 a,
                                                    float4 v, float density) {
    if (wl.count[row] == 0) return make_float3(0.0f, 0.0f, 0.0f);
    float awx = 0.0f, awy = 0.0f, awz = 0.0f;
    each_index(wl, row, walls, [&](uint32_t e, float4 q) {
        float3 r = pair_offset<REL>(p, a, q, e);
        float g = fast_factor(p, fl2(r.x, r.y, r.z));
        awx = fmaf(-r.x, g, awx);
        awy = fmaf(-r.y, g, awy);
        awz = fmaf(-r.z, g, awz);
    });
    float l2 = fl2(awx, awy, awz);
    float nx = 0.0f, ny = 0.0f, nz = 0.0f;
    if (l2 > 0.0f && l2 < FLT_MAX) {
        float inv = rsqrtf(l2);
        nx = awx * inv;
        ny = awy * inv;
        nz = awz * inv;
    }
    float k = fminf(fmaf(v.x, nx, fmaf(v.y, ny, v.z * nz)), 0.0f);
    float ix = nx * k, iy = ny * k, iz = nz * k;
    float px = 0.0f, py = 0.0f, pz = 0.0f;
    float c = -wall_visc * p.mass / density;
    each_index(wl, row, walls, [&](uint32_t e, float4 q) {
        float3 r = pair_offset<REL>(p, a, q, e);
        float toward = fmaf(ix, r.x, fmaf(iy, r.y, iz * r.z));
        if (toward < 0.0f) {
            float l2r = fl2(r.x, r.y, r.z);
            float s = c * toward / (l2r + p.soften) * fast_factor(p, l2r);
            px = fmaf(-r.x, s, px);
            py = fmaf(-r.y, s, py);
            pz = fmaf(-r.z, s, pz);
        }
    });
    return make_float3(px, py, pz);
}

// ---- advance (step.rs:305-339) ----------------------------------------------------------------

__device__ __forceinline__ void clamp_into(const Params& p, float& nx, float& ny, float& nz, float4& v,
                                           uint32_t& held) {
    if (!p.has_bounds) return;
    float ix = fminf(fmaxf(nx, p.low_in.x), p.high_in.x);
    float iy = fminf(fmaxf(ny, p.low_in.y), p.high_in.y);
    float iz = fminf(fmaxf(nz, p.low_in.z), p.high_in.z);
    if (ix != nx || iy != ny || iz != nz) {
        float cx = fminf(fmaxf(nx, p.low.x), p.high.x);
        float cy = fminf(fmaxf(ny, p.low.y), p.high.y);
        float cz = fminf(fmaxf(nz, p.low.z), p.high.z);
        if (cx != nx || cy != ny || cz != nz) held += 1;
        if (ix != nx) v.x = 0.0f;
        if (iy != ny) v.y = 0.0f;
        if (iz != nz) v.z = 0.0f;
        nx = ix;
        ny = iy;
        nz = iz;
    }
}

__device__ __forceinline__ void advance_fast(const Params& p, float dt, float4& a, float4& v, uint32_t& held,
                                             uint32_t& bad) {
    float nx = fmaf(v.x, dt, a.x), ny = fmaf(v.y, dt, a.y), nz = fmaf(v.z, dt, a.z);
    clamp_into(p, nx, ny, nz, v, held);
    if (!(isfinite(nx) && isfinite(ny) && isfinite(nz) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) bad = 1;
    a.x = nx;
    a.y = ny;
    a.z = nz;
}

// One axis of a cell-relative position moved by d: the offset stays in [0, r), the cell follows.
__device__ __forceinline__ void renormalise(float r, float& o, int& c) {
    if (o >= 0.0f && o < r) return;
    float k = floorf(o / r);
    c += int(k);
    o = fmaf(-k, r, o);
    if (o < 0.0f) {  // rounding at the edge
        o += r;
        c -= 1;
    }
    if (o >= r) {
        o -= r;
        c += 1;
    }
}

// The advance in cell-relative form: offsets move by v dt; the container clamp compares the
// position rebuilt in double with the bounds (f32 absolute coordinates lose the offsets' bits).
__device__ __forceinline__ void advance_rel(const Params& p, float dt, float4& a, int4& c, float4& v, uint32_t& held,
                                            uint32_t& bad) {
    float ox = fmaf(v.x, dt, a.x), oy = fmaf(v.y, dt, a.y), oz = fmaf(v.z, dt, a.z);
    if (p.has_bounds) {
        const double r = p.radius;
        double x = double(c.x) * r + ox, y = double(c.y) * r + oy, z = double(c.z) * r + oz;
        double ix = fmin(fmax(x, (double)p.low_in.x), (double)p.high_in.x);
        double iy = fmin(fmax(y, (double)p.low_in.y), (double)p.high_in.y);
        double iz = fmin(fmax(z, (double)p.low_in.z), (double)p.high_in.z);
        if (ix != x || iy != y || iz != z) {
            double cx = fmin(fmax(x, (double)p.low.x), (double)p.high.x);
            double cy = fmin(fmax(y, (double)p.low.y), (double)p.high.y);
            double cz = fmin(fmax(z, (double)p.low.z), (double)p.high.z);
            if (cx != x || cy != y || cz != z) held += 1;
            if (ix != x) {
                v.x = 0.0f;
                ox = float(ix - double(c.x) * r);
            }
            if (iy != y) {
                v.y = 0.0f;
                oy = float(iy - double(c.y) * r);
            }
            if (iz != z) {
                v.z = 0.0f;
                oz = float(iz - double(c.z) * r);
            }
        }
    }
    if (!(isfinite(ox) && isfinite(oy) && isfinite(oz) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) {
        bad = 1;
    } else {
        renormalise(p.radius, ox, c.x);
        renormalise(p.radius, oy, c.y);
        renormalise(p.radius, oz, c.z);
    }
    a.x = ox;
    a.y = oy;
    a.z = oz;
}

__device__ __forceinline__ void fold_stats(Status* st, bool valid, int3 c, float speed, uint32_t held, uint32_t bad) {
    int lox = valid ? c.x : INT_MAX, loy = valid ? c.y : INT_MAX, loz = valid ? c.z : INT_MAX;
    int hix = valid ? c.x : INT_MIN, hiy = valid ? c.y : INT_MIN, hiz = valid ? c.z : INT_MIN;
    uint32_t sb = (valid && speed > 0.0f) ? __float_as_uint(speed) : 0u;
    lox = block_reduce(lox, MinI(), INT_MAX);
    loy = block_reduce(loy, MinI(), INT_MAX);
    loz = block_reduce(loz, MinI(), INT_MAX);
    hix = block_reduce(hix, MaxI(), INT_MIN);
    hiy = block_reduce(hiy, MaxI(), INT_MIN);
    hiz = block_reduce(hiz, MaxI(), INT_MIN);
    sb = block_reduce(sb, MaxU(), 0u);
    held = block_reduce(held, SumU(), 0u);
    bad = block_reduce(bad, MaxU(), 0u);
    if (threadIdx.x == 0) {
        if (lox != INT_MAX) {
            atomicMin(&st->cell_lo[0], lox);
            atomicMin(&st->cell_lo[1], loy);
            atomicMin(&st->cell_lo[2], loz);
            atomicMax(&st->cell_hi[0], hix);
            atomicMax(&st->cell_hi[1], hiy);
            atomicMax(&st->cell_hi[2], hiz);
        }
        if (sb) atomicMax(&st->vmax_bits, sb);
        if (held) atomicAdd(&st->held, held);
        if (bad) atomicMax(&st->nonfinite, 1u);
    }
}

__device__ __forceinline__ void record_clamp(float4* vel_pre, uint32_t i, float4 pre, float4 v) {
    if (!vel_pre) return;
    uint32_t flags = (v.x != pre.x ? 1u : 0u) | (v.y != pre.y ? 2u : 0u) | (v.z != pre.z ? 4u : 0u);
    pre.w = __uint_as_float(flags);
    vel_pre[i] = pre;
}

// ---- WCSPH forces, velocity update, advance (step.rs:159-223, 305-339) ---------------------

template <bool REL>
__global__ void __launch_bounds__(kBlock) k_wcsph_force_fast(Params p, const StepConsts* __restrict__ sc,
                                                             PairLists fpl, PairLists wpl,
                                                             const float4* __restrict__ pos,
                                                             const int4* __restrict__ cells,
                                                             const float4* __restrict__ vel,
                                                             const float* __restrict__ rho,
                                                             const float* __restrict__ press,
                                                             const float* __restrict__ scaled,
                                                             const float4* __restrict__ walls,
                                                             float4* __restrict__ pos_out, int4* __restrict__ cells_out,
                                                             float4* __restrict__ vel_out, Status* st,
                                                             float4* __restrict__ vel_pre) {
    IndexLists fl = index_lists(fpl), wl = index_lists(wpl);
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = row < p.n ? fpl.particle(row) : row;  // row of the walk order, its particle
    bool valid = i < p.n;
    int3 nc = make_int3(0, 0, 0);
    float speed = 0.0f;
    uint32_t held = 0, bad = 0;
    if (valid) {
        const float dt = sc->dt;
        const float visc2 = -2.0f * sc->viscosity;
        float4 a = pos[i];
        float4 v = vel[i];
        float density = rho[i];
        float own = scaled[i];
        float px = 0.0f, py = 0.0f, pz = 0.0f;
        each_index2(fl, row, pos, vel, [&](uint32_t e, float4 q, float4 w) {
            float3 r = pair_offset<REL>(p, a, q, e);
            float squared = fl2(r.x, r.y, r.z);
            if (squared <= 0.0f) return;
            float g = fast_factor(p, squared);
            float toward = fminf(fmaf(v.x - w.x, r.x, fmaf(v.y - w.y, r.y, (v.z - w.z) * r.z)), 0.0f);
            float damp = visc2 * toward / ((squared + p.soften) * (density + __ldg(&rho[e & kIndexMask])));
            float s = g * p.mass * (own + __ldg(&scaled[e & kIndexMask]) + damp);
            px = fmaf(-r.x, s, px);
            py = fmaf(-r.y, s, py);
            pz = fmaf(-r.z, s, pz);
        });
        float mirrored = p.mass * (own + press[i] * p.inv_rest_sq);
        each_index(wl, row, walls, [&](uint32_t e, float4 q) {
            float3 r = pair_offset<REL>(p, a, q, e);
            float s = fast_factor(p, fl2(r.x, r.y, r.z)) * mirrored;
            px = fmaf(-r.x, s, px);
            py = fmaf(-r.y, s, py);
            pz = fmaf(-r.z, s, pz);
        });
        float3 wv = wall_viscous_fast<REL>(p, sc->wall_viscosity, wl, walls, row, a, v, density);
        v.x = fmaf(px + wv.x + p.gravity.x, dt, v.x);
        v.y = fmaf(py + wv.y + p.gravity.y, dt, v.y);
        v.z = fmaf(pz + wv.z + p.gravity.z, dt, v.z);
        float4 pre = v;
        if (REL) {
            int4 c = cells[i];
            advance_rel(p, dt, a, c, v, held, bad);
            cells_out[i] = c;
            nc = make_int3(c.x, c.y, c.z);
        } else {
            advance_fast(p, dt, a, v, held, bad);
            nc = cell_of(p, a.x, a.y, a.z);
        }
        record_clamp(vel_pre, i, pre, v);
        pos_out[i] = a;
        vel_out[i] = v;
        speed = sqrtf(dot3(v.x, v.y, v.z, v.x, v.y, v.z));
        if (!(speed == speed)) speed = 0.0f;
    }
    fold_stats(st, valid, nc, speed, held, bad);
}

// ---- DFSPH: density rate and stiffness, push_apart, viscosity, advance ------------------------

template <int WHICH, bool REL, class Src>
__device__ __forceinline__ void rate_particle_fast(const Params& p, const StepConsts* __restrict__ sc,
                                                   const IndexLists& fl, const IndexLists& wl, uint32_t i, uint32_t row,
                                                   const Src& src, const float4* __restrict__ pos,
                                                   const float4* __restrict__ vel, const float* __restrict__ rho,
                                                   const float* __restrict__ alpha,
                                                   const float4* __restrict__ walls, float* __restrict__ kappa,
                                                   SolveRec rec, uint32_t slot, double& err, uint32_t& loaded) {
    const float dt = sc->dt;
    float4 a = pos[i];
    float4 v = vel[i];
    float rate = 0.0f;
    each_index2_from(fl, row, src, [&](uint32_t e, float4 q, float4 w) {
        float3 r = pair_offset<REL>(p, a, q, e);
        float g = fast_factor(p, fl2(r.x, r.y, r.z));
        rate = fmaf(g, fmaf(v.x - w.x, r.x, fmaf(v.y - w.y, r.y, (v.z - w.z) * r.z)), rate);
    });
    each_index(wl, row, walls, [&](uint32_t e, float4 q) {
        float3 r = pair_offset<REL>(p, a, q, e);
        float g = fast_factor(p, fl2(r.x, r.y, r.z));
        rate = fmaf(g, fmaf(v.x, r.x, fmaf(v.y, r.y, v.z * r.z)), rate);
    });
    rate = rate * p.mass;
    if (rec.rate) {
        size_t at = size_t(slot) * p.n + i;
        rec.rate[at] = rate;
        rec.vel[at] = v;
    }
    float target, error;
    if (WHICH == 1) {
        float over = fmaxf(fmaf(dt, rate, rho[i]) - p.rest, 0.0f);
        target = over / sc->dt_sq;
        error = over * p.inv_rest;
    } else {
        float r = fl.count[row] + wl.count[row] < 20u ? 0.0f : fmaxf(rate, 0.0f);
        target = r / dt;
        error = dt * r * p.inv_rest;
    }
    // the stiffness goes into the position's spare lane
    kappa[4 * (size_t)i + 3] = target * alpha[i];
    err = (double)error;
    loaded = error > 0.0f ? 1u : 0u;
}

template <int WHICH, bool REL>
__global__ void __launch_bounds__(kBlock) k_rate_fast(Params p, const StepConsts* __restrict__ sc, PairLists fpl,
                                                      PairLists wpl, const float4* __restrict__ pos,
                                                      const float4* __restrict__ vel, const float* __restrict__ rho,
                                                      const float* __restrict__ alpha,
                                                      const float4* __restrict__ walls, float* __restrict__ kappa,
                                                      DD* __restrict__ partial,
                                                      uint32_t* __restrict__ partial_loaded, Status* st,
                                                      SolveRec rec, unsigned long long loop) {
    if (__ldcg(&st->settled)) return;
    const uint32_t slot = rec.rate ? __ldcg(&st->iterations) : 0u;
    IndexLists fl = index_lists(fpl), wl = index_lists(wpl);
    DD acc{0.0, 0.0};
    uint32_t loaded = 0;
    // rows of the walk order, a grid's width apart (one each when the grid covers them all)
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < p.n; row += gridDim.x * blockDim.x) {
        double err = 0.0;
        uint32_t one = 0;
        rate_particle_fast<WHICH, REL>(p, sc, fl, wl, fpl.particle(row), row, FromGlobalF{pos, vel}, pos, vel, rho,
                                       alpha, walls, kappa, rec, slot, err, one);
        acc = dd_add(acc, DD{err, 0.0});
        loaded += one;
    }
    residual_finish<WHICH>(p, st, partial, partial_loaded, acc, loaded, loop);
}

template <bool REL, class Src>
__device__ __forceinline__ void push_particle_fast(const Params& p, const StepConsts* __restrict__ sc,
                                                   const IndexLists& fl, const IndexLists& wl, uint32_t i, uint32_t row,
                                                   const Src& src, const float4* __restrict__ pos,
                                                   float4* __restrict__ vel, const float4* __restrict__ walls,
                                                   float* __restrict__ applied) {
    const float mdt = p.mass * sc->dt;
    float4 a = pos[i];
    float own = a.w;
    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
    each_index_from(fl, row, src, [&](uint32_t e, float4 q) {
        float3 r = pair_offset<REL>(p, a, q, e);
        float s = fast_factor(p, fl2(r.x, r.y, r.z)) * (own + q.w);
        cx = fmaf(-r.x, s, cx);
        cy = fmaf(-r.y, s, cy);
        cz = fmaf(-r.z, s, cz);
    });
    each_index(wl, row, walls, [&](uint32_t e, float4 q) {
        float3 r = pair_offset<REL>(p, a, q, e);
        float s = fast_factor(p, fl2(r.x, r.y, r.z)) * own;
        cx = fmaf(-r.x, s, cx);
        cy = fmaf(-r.y, s, cy);
        cz = fmaf(-r.z, s, cz);
    });
    float4 v = vel[i];
    v.x = fmaf(cx, mdt, v.x);
    v.y = fmaf(cy, mdt, v.y);
    v.z = fmaf(cz, mdt, v.z);
    vel[i] = v;
    if (applied) applied[2 * (size_t)i] = fmaf(own, sc->dt, applied[2 * (size_t)i]);
}

template <bool REL>
__global__ void __launch_bounds__(kBlock) k_push_fast(Params p, const StepConsts* __restrict__ sc, PairLists fpl,
                                                      PairLists wpl, const float4* __restrict__ pos,
                                                      float4* __restrict__ vel, const float4* __restrict__ walls,
                                                      Status* st, float* __restrict__ applied,
                                                      unsigned long long loop) {
    loop_bound(p, st, loop);
    if (__ldcg(&st->settled)) return;
    IndexLists fl = index_lists(fpl), wl = index_lists(wpl);
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = row < p.n ? fpl.particle(row) : row;  // row of the walk order, its particle
    if (i >= p.n) return;
    push_particle_fast<REL>(p, sc, fl, wl, i, row, FromGlobalF{pos, nullptr}, pos, vel, walls, applied);
}

template <bool REL>
__global__ void __launch_bounds__(kBlock) k_viscous_fast(Params p, const StepConsts* __restrict__ sc,
                                                         PairLists fpl, PairLists wpl,
                                                         const float4* __restrict__ pos,
                                                         const float4* __restrict__ vel,
                                                         const float* __restrict__ rho,
                                                         const float4* __restrict__ walls,
                                                         float4* __restrict__ vel_out) {
    IndexLists fl = index_lists(fpl), wl = index_lists(wpl);
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = row < p.n ? fpl.particle(row) : row;  // row of the walk order, its particle
    if (i >= p.n) return;
    const float dt = sc->dt;
    const float visc2 = -2.0f * sc->viscosity * p.mass;
    float4 a = pos[i];
    float4 v = vel[i];
    float density = rho[i];
    float px = 0.0f, py = 0.0f, pz = 0.0f;
    each_index2(fl, row, pos, vel, [&](uint32_t e, float4 q, float4 w) {
        uint32_t j = e & kIndexMask;
        if (j == i) return;
        float3 r = pair_offset<REL>(p, a, q, e);
        float toward = fmaf(v.x - w.x, r.x, fmaf(v.y - w.y, r.y, (v.z - w.z) * r.z));
        if (toward < 0.0f) {
            float l2 = fl2(r.x, r.y, r.z);
            float s = visc2 * toward / ((l2 + p.soften) * (density + __ldg(&rho[j]))) * fast_factor(p, l2);
            px = fmaf(-r.x, s, px);
            py = fmaf(-r.y, s, py);
            pz = fmaf(-r.z, s, pz);
        }
    });
    float3 wv = wall_viscous_fast<REL>(p, sc->wall_viscosity, wl, walls, row, a, v, density);
    v.x = fmaf(px + wv.x + p.gravity.x, dt, v.x);
    v.y = fmaf(py + wv.y + p.gravity.y, dt, v.y);
    v.z = fmaf(pz + wv.z + p.gravity.z, dt, v.z);
    vel_out[i] = v;
}

// DFSPH advance of cell-relative positions (the absolute one is k_advance in kernels.cu)
__global__ void k_advance_rel(Params p, const StepConsts* __restrict__ sc, const float4* __restrict__ pos_in,
                              const int4* __restrict__ cells_in, float4* __restrict__ pos_out,
                              int4* __restrict__ cells_out, float4* __restrict__ vel, Status* st,
                              float4* __restrict__ vel_pre) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < p.n;
    int3 nc = make_int3(0, 0, 0);
    float speed = 0.0f;
    uint32_t held = 0, bad = 0;
    if (valid) {
        float4 a = pos_in[i];
        int4 c = cells_in[i];
        float4 v = vel[i];
        float4 pre = v;
        advance_rel(p, sc->dt, a, c, v, held, bad);
        record_clamp(vel_pre, i, pre, v);
        pos_out[i] = a;
        cells_out[i] = c;
        vel[i] = v;
        nc = make_int3(c.x, c.y, c.z);
        speed = sqrtf(dot3(v.x, v.y, v.z, v.x, v.y, v.z));
        if (!(speed == speed)) speed = 0.0f;
    }
    fold_stats(st, valid, nc, speed, held, bad);
}

// ---- cell-relative positions in and out -----------------------------------------------------

// absolute f32 positions -> offset in [0, r) and cell, cell = floor(x / r) as cell_of has it
__global__ void k_to_relative(Params p, uint32_t n, const float* __restrict__ xyz, const float4* __restrict__ abs4,
                              float4* __restrict__ pos, int4* __restrict__ cells, uint32_t* bad) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x, y, z;
    if (xyz) {
        x = xyz[3 * i];
        y = xyz[3 * i + 1];
        z = xyz[3 * i + 2];
    } else {
        float4 q = abs4[i];
        x = q.x;
        y = q.y;
        z = q.z;
    }
    if (bad && !(isfinite(x) && isfinite(y) && isfinite(z))) atomicAdd(bad, 1u);
    int3 c = cell_of(p, x, y, z);
    const double r = p.radius;
    float ox = float(double(x) - double(c.x) * r), oy = float(double(y) - double(c.y) * r),
          oz = float(double(z) - double(c.z) * r);
    renormalise(p.radius, ox, c.x);
    renormalise(p.radius, oy, c.y);
    renormalise(p.radius, oz, c.z);
    pos[i] = make_float4(ox, oy, oz, 0.0f);
    cells[i] = make_int4(c.x, c.y, c.z, 0);
}

// offset and cell -> absolute f32 positions, xyz triples
__global__ void k_from_relative(Params p, uint32_t n, const float4* __restrict__ pos, const int4* __restrict__ cells,
                                float* __restrict__ xyz) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 a = pos[i];
    int4 c = cells[i];
    const double r = p.radius;
    xyz[3 * i] = float(double(c.x) * r + a.x);
    xyz[3 * i + 1] = float(double(c.y) * r + a.y);
    xyz[3 * i + 2] = float(double(c.z) * r + a.z);
}

// bounding box of cells and fastest speed of a cell-relative state
__global__ void k_state_stats_rel(Params p, const int4* __restrict__ cells, const float4* __restrict__ vel,
                                  Status* st) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < p.n;
    int3 c = make_int3(0, 0, 0);
    float speed = 0.0f;
    if (valid) {
        int4 c4 = cells[i];
        c = make_int3(c4.x, c4.y, c4.z);
        float4 v = vel[i];
        speed = sqrtf(dot3(v.x, v.y, v.z, v.x, v.y, v.z));
        if (!(speed == speed)) speed = 0.0f;
    }
    fold_stats(st, valid, c, speed, 0u, 0u);
}

// neighbour lists on demand, cell-relative (k_list_count / k_list_fill in kernels.cu)
__global__ void k_list_rel(Params p, GridDev g, const float4* __restrict__ pos, const int4* __restrict__ cells,
                           const float4* __restrict__ pts, const uint32_t* __restrict__ start, uint32_t* out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    float4 a = pos[i];
    int4 c4 = cells[i];
    uint32_t k = start ? start[i] : 0u, c = 0;
    each_near_rel(p, g, pts, make_int3(c4.x, c4.y, c4.z), a,
                  [&](uint32_t j, float4, int, int, int, float, float, float) {
                      if (start) out[k++] = j;
                      else ++c;
                  });
    if (!start) out[i] = c;
}

// ---- launchers ------------------------------------------------------------------------------

static inline uint32_t fast_blocks(uint32_t n) {
    note_launch();
    return (n + kBlock - 1) / kBlock;
}

// The FAST check on grids no larger than the SMs hold at once (as the EXACT one: its last block
// then sums fewer partials); k_rate_fast<which, rel> at [which * 2 + rel], 0 until looked up.
static std::atomic<uint32_t> g_fast_resident[4] = {0, 0, 0, 0};

void prepare_fast_grids() {
    if (g_fast_resident[3].load()) return;
    int dev = 0, sms = 0, per[4] = {0, 0, 0, 0};
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[0], k_rate_fast<0, false>, kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[1], k_rate_fast<0, true>, kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[2], k_rate_fast<1, false>, kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[3], k_rate_fast<1, true>, kBlock, 0);
    for (int k = 0; k < 4; ++k) g_fast_resident[k].store(uint32_t(std::max(per[k], 0) * std::max(sms, 0)));
}

void launch_density_fast(const Params& p, const GridDev& fg, const GridDev& wg, const float4* pos, const int4* cells,
                         const float4* walls, const PairLists& fl, const PairLists& wl, float* rho, float* press,
                         float* scaled, float* alpha, Status* st, cudaStream_t s) {
    if (!p.n) return;
    uint32_t nb = fast_blocks(p.n);
    if (cells) {
        if (p.solver == 0)
            k_density_fast<0, true><<<nb, kBlock, 0, s>>>(p, fg, wg, pos, cells, walls, fl, wl, rho, press, scaled,
                                                           alpha, st);
        else
            k_density_fast<1, true><<<nb, kBlock, 0, s>>>(p, fg, wg, pos, cells, walls, fl, wl, rho, press, scaled,
                                                           alpha, st);
    } else {
        if (p.solver == 0)
            k_density_fast<0, false><<<nb, kBlock, 0, s>>>(p, fg, wg, pos, cells, walls, fl, wl, rho, press, scaled,
                                                            alpha, st);
        else
            k_density_fast<1, false><<<nb, kBlock, 0, s>>>(p, fg, wg, pos, cells, walls, fl, wl, rho, press, scaled,
                                                            alpha, st);
    }
}

void launch_wcsph_force_fast(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                             const float4* pos, const int4* cells, const float4* vel, const float* rho,
                             const float* press, const float* scaled, const float4* walls, float4* pos_out,
                             int4* cells_out, float4* vel_out, Status* st, float4* vel_pre, cudaStream_t s) {
    if (!p.n) return;
    uint32_t nb = fast_blocks(p.n);
    if (cells)
        k_wcsph_force_fast<true><<<nb, kBlock, 0, s>>>(p, sc, fl, wl, pos, cells, vel, rho, press, scaled, walls,
                                                       pos_out, cells_out, vel_out, st, vel_pre);
    else
        k_wcsph_force_fast<false><<<nb, kBlock, 0, s>>>(p, sc, fl, wl, pos, cells, vel, rho, press, scaled, walls,
                                                        pos_out, cells_out, vel_out, st, vel_pre);
}

void launch_rate_fast(int which, bool rel, const Params& p, const StepConsts* sc, const PairLists& fl,
                      const PairLists& wl, float4* pos, const float4* vel, const float* rho, const float* alpha,
                      const float4* walls, void* partials, Status* st, SolveRec rec, cudaStream_t s,
                      unsigned long long loop) {
    if (!p.n) return;
    uint32_t nb = fast_blocks(p.n);
    const uint32_t resident = g_fast_resident[which * 2 + (rel ? 1 : 0)].load();
    DD* part = static_cast<DD*>(partials);
    uint32_t* loaded = reinterpret_cast<uint32_t*>(part + nb);  // the partials' room: a block a 256 rows
    if (resident && resident < nb) nb = resident;
    float* kw = reinterpret_cast<float*>(pos);
    if (which == 0 && rel)
        k_rate_fast<0, true><<<nb, kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, alpha, walls, kw, part, loaded, st,
                                                   rec, loop);
    else if (which == 0)
        k_rate_fast<0, false><<<nb, kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, alpha, walls, kw, part, loaded, st,
                                                    rec, loop);
    else if (rel)
        k_rate_fast<1, true><<<nb, kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, alpha, walls, kw, part, loaded, st,
                                                   rec, loop);
    else
        k_rate_fast<1, false><<<nb, kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, alpha, walls, kw, part, loaded, st,
                                                    rec, loop);
}

void launch_push_fast(bool rel, const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                      const float4* pos, float4* vel, const float4* walls, Status* st, float* applied,
                      cudaStream_t s, unsigned long long loop) {
    if (!p.n) return;
    if (rel) k_push_fast<true><<<fast_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, walls, st, applied, loop);
    else k_push_fast<false><<<fast_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, walls, st, applied, loop);
}

void launch_viscous_fast(bool rel, const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                         const float4* pos, const float4* vel, const float* rho, const float4* walls,
                         float4* vel_out, cudaStream_t s) {
    if (!p.n) return;
    if (rel)
        k_viscous_fast<true><<<fast_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, walls, vel_out);
    else
        k_viscous_fast<false><<<fast_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, walls, vel_out);
}

void launch_advance_rel(const Params& p, const StepConsts* sc, const float4* pos_in, const int4* cells_in,
                        float4* pos_out, int4* cells_out, float4* vel, Status* st, float4* vel_pre, cudaStream_t s) {
    if (p.n)
        k_advance_rel<<<fast_blocks(p.n), kBlock, 0, s>>>(p, sc, pos_in, cells_in, pos_out, cells_out, vel, st,
                                                          vel_pre);
}

void launch_to_relative(const Params& p, uint32_t n, const float* xyz, const float4* abs4, float4* pos, int4* cells,
                        cudaStream_t s, uint32_t* bad) {
    if (n) k_to_relative<<<fast_blocks(n), kBlock, 0, s>>>(p, n, xyz, abs4, pos, cells, bad);
}

void launch_from_relative(const Params& p, uint32_t n, const float4* pos, const int4* cells, float* xyz,
                          cudaStream_t s) {
    if (n) k_from_relative<<<fast_blocks(n), kBlock, 0, s>>>(p, n, pos, cells, xyz);
}

void launch_state_stats_rel(const Params& p, const int4* cells, const float4* vel, Status* st, cudaStream_t s) {
    if (p.n) k_state_stats_rel<<<fast_blocks(p.n), kBlock, 0, s>>>(p, cells, vel, st);
}

void launch_list_rel(const Params& p, const GridDev& g, const float4* pos, const int4* cells, const float4* pts,
                     const uint32_t* start, uint32_t* out, cudaStream_t s) {
    if (p.n) k_list_rel<<<fast_blocks(p.n), kBlock, 0, s>>>(p, g, pos, cells, pts, start, out);
}

}  // namespace slf
