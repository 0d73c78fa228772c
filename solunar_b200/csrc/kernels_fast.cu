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
#include <cfloat>
#include <climits>

#include "fluid_device.cuh"
#include "launch.h"
#include "reduce.cuh"

namespace slf {

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

// f(j, q) for each listed neighbour, four entries and their gathers ahead.
template <class F>
__device__ __forceinline__ void each_index(const IndexLists& l, uint32_t i, const float4* __restrict__ pts, F&& f) {
    uint32_t n = l.count[i];
    if (n > l.cap) n = l.cap;
    if (n == 0) return;
    const uint32_t* __restrict__ base = l.idx + l.at(i, 0);
    for (uint32_t k = 0; k < n; k += 4) {
        uint32_t j[4];
        float4 q[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) j[u] = __ldg(base + size_t(k + u < n ? k + u : n - 1) * 32u);
#pragma unroll
        for (int u = 0; u < 4; ++u) q[u] = __ldg(&pts[j[u]]);
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k + u < n) f(j[u], q[u]);
    }
}

template <class F>
__device__ __forceinline__ void each_index2(const IndexLists& l, uint32_t i, const float4* __restrict__ pts,
                                            const float4* __restrict__ more, F&& f) {
    uint32_t n = l.count[i];
    if (n > l.cap) n = l.cap;
    if (n == 0) return;
    const uint32_t* __restrict__ base = l.idx + l.at(i, 0);
    for (uint32_t k = 0; k < n; k += 4) {
        uint32_t j[4];
        float4 q[4], w[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) j[u] = __ldg(base + size_t(k + u < n ? k + u : n - 1) * 32u);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            q[u] = __ldg(&pts[j[u]]);
            w[u] = __ldg(&more[j[u]]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k + u < n) f(j[u], q[u], w[u]);
    }
}

// ---- densities and lists (mod.rs:621-675; step.rs:147-172; dfsph.rs:108-163) ---------------

template <int SOLVER>
__global__ void __launch_bounds__(kBlock) k_density_fast(Params p, GridDev fg, GridDev wg,
                                                         const float4* __restrict__ pos,
                                                         const float4* __restrict__ walls, PairLists fpl,
                                                         PairLists wpl, float* __restrict__ rho,
                                                         float* __restrict__ press, float* __restrict__ scaled,
                                                         float* __restrict__ alpha, Status* st) {
    IndexLists fl = index_lists(fpl), wl = index_lists(wpl);
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < p.n;
    uint32_t compressed = 0, longest = 0;
    if (valid) {
        float4 a = pos[i];
        int3 cell = cell_of(p, a.x, a.y, a.z);
        float sum = 0.0f, wsum = 0.0f;
        float sx = 0.0f, sy = 0.0f, sz = 0.0f, squares = 0.0f;
        uint32_t nf = 0, nw = 0;
        each_near(p, fg, pos, cell, a.x, a.y, a.z, [&](uint32_t j, float4 q) {
            float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
            float l2 = fl2(rx, ry, rz);
            sum += fast_value(p, l2);
            if (nf < fl.cap) fl.idx[fl.at(i, nf)] = j;
            ++nf;
            if (SOLVER == 1) {
                float g = fast_factor(p, l2) * p.mass;
                float px = rx * g, py = ry * g, pz = rz * g;
                sx += px;
                sy += py;
                sz += pz;
                squares = fmaf(px, px, fmaf(py, py, fmaf(pz, pz, squares)));
            }
        });
        each_near(p, wg, walls, cell, a.x, a.y, a.z, [&](uint32_t j, float4 q) {
            float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
            float l2 = fl2(rx, ry, rz);
            wsum += fast_value(p, l2);
            if (nw < wl.cap) wl.idx[wl.at(i, nw)] = j;
            ++nw;
            if (SOLVER == 1) {
                float g = fast_factor(p, l2) * p.mass;
                sx = fmaf(rx, g, sx);
                sy = fmaf(ry, g, sy);
                sz = fmaf(rz, g, sz);
            }
        });
        fl.count[i] = nf;
        wl.count[i] = nw;
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

__device__ __forceinline__ float3 wall_viscous_fast(const Params& p, float wall_visc, const IndexLists& wl,
                                                    const float4* __restrict__ walls, uint32_t i, float4 a,
                                                    float4 v, float density) {
    if (wl.count[i] == 0) return make_float3(0.0f, 0.0f, 0.0f);
    float awx = 0.0f, awy = 0.0f, awz = 0.0f;
    each_index(wl, i, walls, [&](uint32_t, float4 q) {
        float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
        float g = fast_factor(p, fl2(rx, ry, rz));
        awx = fmaf(-rx, g, awx);
        awy = fmaf(-ry, g, awy);
        awz = fmaf(-rz, g, awz);
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
    each_index(wl, i, walls, [&](uint32_t, float4 q) {
        float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
        float toward = fmaf(ix, rx, fmaf(iy, ry, iz * rz));
        if (toward < 0.0f) {
            float l2r = fl2(rx, ry, rz);
            float s = c * toward / (l2r + p.soften) * fast_factor(p, l2r);
            px = fmaf(-rx, s, px);
            py = fmaf(-ry, s, py);
            pz = fmaf(-rz, s, pz);
        }
    });
    return make_float3(px, py, pz);
}

// ---- WCSPH forces, velocity update, advance (step.rs:159-223, 305-339) ---------------------

__device__ __forceinline__ void advance_fast(const Params& p, float dt, float4& a, float4& v, uint32_t& held,
                                             uint32_t& bad) {
    float nx = fmaf(v.x, dt, a.x), ny = fmaf(v.y, dt, a.y), nz = fmaf(v.z, dt, a.z);
    if (p.has_bounds) {
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
    if (!(isfinite(nx) && isfinite(ny) && isfinite(nz) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) bad = 1;
    a.x = nx;
    a.y = ny;
    a.z = nz;
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

__global__ void __launch_bounds__(kBlock) k_wcsph_force_fast(Params p, const StepConsts* __restrict__ sc,
                                                             PairLists fpl, PairLists wpl,
                                                             const float4* __restrict__ pos,
                                                             const float4* __restrict__ vel,
                                                             const float* __restrict__ rho,
                                                             const float* __restrict__ press,
                                                             const float* __restrict__ scaled,
                                                             const float4* __restrict__ walls,
                                                             float4* __restrict__ pos_out,
                                                             float4* __restrict__ vel_out, Status* st,
                                                             float4* __restrict__ vel_pre) {
    IndexLists fl = index_lists(fpl), wl = index_lists(wpl);
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
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
        each_index2(fl, i, pos, vel, [&](uint32_t j, float4 q, float4 w) {
            float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
            float squared = fl2(rx, ry, rz);
            if (squared <= 0.0f) return;
            float g = fast_factor(p, squared);
            float toward = fminf(fmaf(v.x - w.x, rx, fmaf(v.y - w.y, ry, (v.z - w.z) * rz)), 0.0f);
            float damp = visc2 * toward / ((squared + p.soften) * (density + __ldg(&rho[j])));
            float s = g * p.mass * (own + __ldg(&scaled[j]) + damp);
            px = fmaf(-rx, s, px);
            py = fmaf(-ry, s, py);
            pz = fmaf(-rz, s, pz);
        });
        float mirrored = p.mass * (own + press[i] * p.inv_rest_sq);
        each_index(wl, i, walls, [&](uint32_t, float4 q) {
            float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
            float s = fast_factor(p, fl2(rx, ry, rz)) * mirrored;
            px = fmaf(-rx, s, px);
            py = fmaf(-ry, s, py);
            pz = fmaf(-rz, s, pz);
        });
        float3 wv = wall_viscous_fast(p, sc->wall_viscosity, wl, walls, i, a, v, density);
        v.x = fmaf(px + wv.x + p.gravity.x, dt, v.x);
        v.y = fmaf(py + wv.y + p.gravity.y, dt, v.y);
        v.z = fmaf(pz + wv.z + p.gravity.z, dt, v.z);
        float4 pre = v;
        advance_fast(p, dt, a, v, held, bad);
        if (vel_pre) {
            uint32_t flags = (v.x != pre.x ? 1u : 0u) | (v.y != pre.y ? 2u : 0u) | (v.z != pre.z ? 4u : 0u);
            pre.w = __uint_as_float(flags);
            vel_pre[i] = pre;
        }
        pos_out[i] = a;
        vel_out[i] = v;
        nc = cell_of(p, a.x, a.y, a.z);
        speed = sqrtf(dot3(v.x, v.y, v.z, v.x, v.y, v.z));
        if (!(speed == speed)) speed = 0.0f;
    }
    fold_stats(st, valid, nc, speed, held, bad);
}

// ---- DFSPH: density rate and stiffness, push_apart, viscosity --------------------------------

template <int WHICH>
__global__ void __launch_bounds__(kBlock) k_rate_fast(Params p, const StepConsts* __restrict__ sc, PairLists fpl,
                                                      PairLists wpl, const float4* __restrict__ pos,
                                                      const float4* __restrict__ vel, const float* __restrict__ rho,
                                                      const float* __restrict__ alpha,
                                                      const float4* __restrict__ walls, float* __restrict__ kappa_w,
                                                      DD* __restrict__ partial,
                                                      uint32_t* __restrict__ partial_loaded, Status* st,
                                                      float* __restrict__ rate_out) {
    if (__ldcg(&st->settled)) return;
    IndexLists fl = index_lists(fpl), wl = index_lists(wpl);
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double err = 0.0;
    uint32_t loaded = 0;
    if (i < p.n) {
        const float dt = sc->dt;
        float4 a = pos[i];
        float4 v = vel[i];
        float rate = 0.0f;
        each_index2(fl, i, pos, vel, [&](uint32_t, float4 q, float4 w) {
            float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
            float g = fast_factor(p, fl2(rx, ry, rz));
            rate = fmaf(g, fmaf(v.x - w.x, rx, fmaf(v.y - w.y, ry, (v.z - w.z) * rz)), rate);
        });
        each_index(wl, i, walls, [&](uint32_t, float4 q) {
            float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
            float g = fast_factor(p, fl2(rx, ry, rz));
            rate = fmaf(g, fmaf(v.x, rx, fmaf(v.y, ry, v.z * rz)), rate);
        });
        rate = rate * p.mass;
        if (rate_out) rate_out[i] = rate;
        float target, error;
        if (WHICH == 1) {
            float over = fmaxf(fmaf(dt, rate, rho[i]) - p.rest, 0.0f);
            target = over / sc->dt_sq;
            error = over * p.inv_rest;
        } else {
            float r = fl.count[i] + wl.count[i] < 20u ? 0.0f : fmaxf(rate, 0.0f);
            target = r / dt;
            error = dt * r * p.inv_rest;
        }
        kappa_w[4 * (size_t)i + 3] = target * alpha[i];
        err = (double)error;
        loaded = error > 0.0f ? 1u : 0u;
    }
    residual_finish<WHICH>(p, st, partial, partial_loaded, err, loaded);
}

__global__ void __launch_bounds__(kBlock) k_push_fast(Params p, const StepConsts* __restrict__ sc, PairLists fpl,
                                                      PairLists wpl, const float4* __restrict__ pos,
                                                      float4* __restrict__ vel, const float4* __restrict__ walls,
                                                      const Status* st) {
    if (__ldcg(&st->settled)) return;
    IndexLists fl = index_lists(fpl), wl = index_lists(wpl);
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const float mdt = p.mass * sc->dt;
    float4 a = pos[i];
    float own = a.w;
    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
    each_index(fl, i, pos, [&](uint32_t, float4 q) {
        float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
        float s = fast_factor(p, fl2(rx, ry, rz)) * (own + q.w);
        cx = fmaf(-rx, s, cx);
        cy = fmaf(-ry, s, cy);
        cz = fmaf(-rz, s, cz);
    });
    each_index(wl, i, walls, [&](uint32_t, float4 q) {
        float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
        float s = fast_factor(p, fl2(rx, ry, rz)) * own;
        cx = fmaf(-rx, s, cx);
        cy = fmaf(-ry, s, cy);
        cz = fmaf(-rz, s, cz);
    });
    float4 v = vel[i];
    v.x = fmaf(cx, mdt, v.x);
    v.y = fmaf(cy, mdt, v.y);
    v.z = fmaf(cz, mdt, v.z);
    vel[i] = v;
}

__global__ void __launch_bounds__(kBlock) k_viscous_fast(Params p, const StepConsts* __restrict__ sc,
                                                         PairLists fpl, PairLists wpl,
                                                         const float4* __restrict__ pos,
                                                         const float4* __restrict__ vel,
                                                         const float* __restrict__ rho,
                                                         const float4* __restrict__ walls,
                                                         float4* __restrict__ vel_out) {
    IndexLists fl = index_lists(fpl), wl = index_lists(wpl);
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const float dt = sc->dt;
    const float visc2 = -2.0f * sc->viscosity * p.mass;
    float4 a = pos[i];
    float4 v = vel[i];
    float density = rho[i];
    float px = 0.0f, py = 0.0f, pz = 0.0f;
    each_index2(fl, i, pos, vel, [&](uint32_t j, float4 q, float4 w) {
        if (j == i) return;
        float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
        float toward = fmaf(v.x - w.x, rx, fmaf(v.y - w.y, ry, (v.z - w.z) * rz));
        if (toward < 0.0f) {
            float l2 = fl2(rx, ry, rz);
            float s = visc2 * toward / ((l2 + p.soften) * (density + __ldg(&rho[j]))) * fast_factor(p, l2);
            px = fmaf(-rx, s, px);
            py = fmaf(-ry, s, py);
            pz = fmaf(-rz, s, pz);
        }
    });
    float3 wv = wall_viscous_fast(p, sc->wall_viscosity, wl, walls, i, a, v, density);
    v.x = fmaf(px + wv.x + p.gravity.x, dt, v.x);
    v.y = fmaf(py + wv.y + p.gravity.y, dt, v.y);
    v.z = fmaf(pz + wv.z + p.gravity.z, dt, v.z);
    vel_out[i] = v;
}

// ---- launchers ------------------------------------------------------------------------------

static inline uint32_t fast_blocks(uint32_t n) {
    note_launch();
    return (n + kBlock - 1) / kBlock;
}

void launch_density_fast(const Params& p, const GridDev& fg, const GridDev& wg, const float4* pos,
                         const float4* walls, const PairLists& fl, const PairLists& wl, float* rho, float* press,
                         float* scaled, float* alpha, Status* st, cudaStream_t s) {
    if (!p.n) return;
    if (p.solver == 0)
        k_density_fast<0><<<fast_blocks(p.n), kBlock, 0, s>>>(p, fg, wg, pos, walls, fl, wl, rho, press, scaled,
                                                               alpha, st);
    else
        k_density_fast<1><<<fast_blocks(p.n), kBlock, 0, s>>>(p, fg, wg, pos, walls, fl, wl, rho, press, scaled,
                                                               alpha, st);
}

void launch_wcsph_force_fast(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                             const float4* pos, const float4* vel, const float* rho, const float* press,
                             const float* scaled, const float4* walls, float4* pos_out, float4* vel_out, Status* st,
                             float4* vel_pre, cudaStream_t s) {
    if (p.n)
        k_wcsph_force_fast<<<fast_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, press, scaled, walls,
                                                               pos_out, vel_out, st, vel_pre);
}

void launch_rate_fast(int which, const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                      float4* pos, const float4* vel, const float* rho, const float* alpha, const float4* walls,
                      void* partials, Status* st, float* rate_out, cudaStream_t s) {
    if (!p.n) return;
    uint32_t nb = fast_blocks(p.n);
    DD* part = static_cast<DD*>(partials);
    uint32_t* loaded = reinterpret_cast<uint32_t*>(part + nb);
    if (which == 0)
        k_rate_fast<0><<<nb, kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, alpha, walls,
                                             reinterpret_cast<float*>(pos), part, loaded, st, rate_out);
    else
        k_rate_fast<1><<<nb, kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, alpha, walls,
                                             reinterpret_cast<float*>(pos), part, loaded, st, rate_out);
}

void launch_push_fast(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                      const float4* pos, float4* vel, const float4* walls, const Status* st, cudaStream_t s) {
    if (p.n) k_push_fast<<<fast_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, walls, st);
}

void launch_viscous_fast(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                         const float4* pos, const float4* vel, const float* rho, const float4* walls,
                         float4* vel_out, cudaStream_t s) {
    if (p.n) k_viscous_fast<<<fast_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, walls, vel_out);
}

}  // namespace slf
