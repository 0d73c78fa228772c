// adjoint.cu -- the hand-written adjoint of the WCSPH substep (step_backward).
//
// The substep (src/fluid/step.rs:144-224, 229-339) maps the sorted state (x, v) to
// x' = clamp(x + v' dt), v' = v + a dt (zeroed where clamped), with
//   a_i = sum_j T(r_ij, u_ij, s_i + s_j, rho_i + rho_j) + walls_i + wall_viscous_i + g,
//   T(r, u, S, R) = -grad W(r) m (S + Pi),  Pi = -nu min(0, u.r) 2 / ((|r|^2 + eps) R),
//   rho_i = m (sum_j W(|r_ij|) + sum_w W(|r_iw|)),  s = p / rho^2,  p = max(0, B (min(rho/rho0, 1.1)^7 - 1)).
// T is odd in (r, u), so the pair's part of the loss, a_i-bar . T_ij + a_j-bar . T_ji, equals
// (a_i-bar - a_j-bar) . T_ij: each particle gathers its own adjoint over its own (symmetric) list,
// with no atomics and no second list.  Neighbour lists are the forward's, fixed for the substep;
// non-smooth points take the branch the forward took.  Particle-level adjoints are FP32; the
// parameter gradients are summed in FP64.
#include <atomic>
#include <cmath>

#include "fluid_device.cuh"
#include "launch.h"
#include "reduce.cuh"

namespace slf {

// How a world's lists hold a neighbour: EXACT lists {index, g} pairs; FAST lists the index in
// the low 26 bits with the cell step to the neighbour in the top six (zero steps for absolute
// positions); cell-relative positions are FAST lists whose steps matter.
enum ListForm : int { kFormFast = 0, kFormExact = 1, kFormCellRelative = 2 };
constexpr uint32_t kEntryIndexMask = (1u << 26) - 1u;

// The entry in slot k: the index (EXACT), or index and step bits (FAST).
__device__ __forceinline__ uint32_t listed_raw(const PairLists& l, int form, uint32_t i, uint32_t k) {
    size_t at = (size_t(i >> 5) * l.cap + k) * 32u + (i & 31u);
    return form == kFormExact ? SLF_LIST_LOAD(&l.e[at]).x : SLF_LIST_LOAD(reinterpret_cast<const uint32_t*>(l.e) + at);
}
__device__ __forceinline__ uint32_t entry_index(uint32_t e, int form) {
    return form == kFormExact ? e : (e & kEntryIndexMask);
}
__device__ __forceinline__ uint32_t listed(const PairLists& l, int form, uint32_t i, uint32_t k) {
    return entry_index(listed_raw(l, form, i, k), form);
}

// x_i - x_j from particle i's stored position xi and neighbour q's, given the entry e: with
// cell-relative positions both are offsets from their cells and the entry's step (c_j - c_i)
// restores the pair's offset as the forward pass forms it, (o_i - o_j) - step r.
__device__ __forceinline__ float3 pair_off(const Params& p, int form, float3 xi, float4 q, uint32_t e) {
    if (form != kFormCellRelative) return make_float3(xi.x - q.x, xi.y - q.y, xi.z - q.z);
    float dx = float(int((e >> 26) & 3u) - 1), dy = float(int((e >> 28) & 3u) - 1),
          dz = float(int((e >> 30) & 3u) - 1);
    return make_float3(fmaf(-dx, p.radius, xi.x - q.x), fmaf(-dy, p.radius, xi.y - q.y),
                       fmaf(-dz, p.radius, xi.z - q.z));
}

__device__ __forceinline__ uint32_t listed_count(const PairLists& l, uint32_t i) {
    uint32_t n = l.count[i];
    return n < l.cap ? n : l.cap;
}

// 1/|r| from d2 = r.r through the reciprocal square root (a few ulp, as FAST arithmetic allows);
// 0 below the smallest normal float, where the pair counts as coincident and adds nothing (the
// hardware flushes such inputs, and 1/0 would turn the pair's zero terms into NaN)
__device__ __forceinline__ float inv_length(float d2) { return d2 >= 1.17549435e-38f ? rsqrtf(d2) : 0.0f; }

// gradient factor g(d) = slope(d) / d = grad_scale (1 - d/r)^3 and its derivative in d
__device__ __forceinline__ void grad_factor(const Params& p, float d, float& g, float& gp) {
    float om = 1.0f - d * p.inv_radius;
    if (om <= 0.0f) {
        g = gp = 0.0f;
        return;
    }
    g = p.grad_scale * om * om * om;
    gp = -3.0f * p.grad_scale * om * om * p.inv_radius;
}

// Walks i's list four entries at a time: gather(j) for all four first, so their loads are in
// flight together, then body(j, gathered, e) for each in list order (the sums keep their order),
// e the raw entry (its cell step for pair_off).
// PREFETCH: the next four entries are requested before the bodies run (past the end the last
// entry is read again and not used); walks that gather several records a neighbour skip it, as
// the registers it holds cost them occupancy.
template <class G, bool PREFETCH = true, class Gather, class Body>
__device__ __forceinline__ void walk4(const PairLists& l, int form, uint32_t i, Gather&& gather, Body&& body) {
    uint32_t n = listed_count(l, i);
    if (n == 0) return;
    uint32_t e[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) e[u] = listed_raw(l, form, i, u < (int)n ? u : n - 1);
    for (uint32_t k = 0; k < n; k += 4) {
        G g[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) g[u] = gather(entry_index(e[u], form));
        uint32_t next[4];
        if (PREFETCH) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                uint32_t kk = k + 4 + u;
                next[u] = listed_raw(l, form, i, kk < n ? kk : n - 1);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k + u < n) body(entry_index(e[u], form), g[u], e[u]);
        if (!PREFETCH) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                uint32_t kk = k + 4 + u;
                next[u] = listed_raw(l, form, i, kk < n ? kk : n - 1);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) e[u] = next[u];
    }
}

// Walks row's entries in both forms at once, U at a time: each pair's gradient G and index
// (PairLists::gv) and its factor g = slope(d) / d (the {index, g} entry); gather(j) for all U
// first, then body(G, g, gathered) in list order.
template <class T, int U, class Gather, class Body>
__device__ __forceinline__ void walk_gradients_g(const PairLists& l, uint32_t row, Gather&& gather, Body&& body) {
    uint32_t n = listed_count(l, row);
    if (n == 0) return;
    const float4* gb = l.gv + l.at(row, 0);
    const uint2* eb = l.e + l.at(row, 0);
    for (uint32_t k = 0; k < n; k += U) {
        float4 G[U];
        float g[U];
        T q[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            uint32_t kk = k + u < n ? k + u : n - 1;
            G[u] = SLF_LIST_LOAD(gb + size_t(kk) * 32u);
            g[u] = __uint_as_float(SLF_LIST_LOAD(eb + size_t(kk) * 32u).y);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) q[u] = gather(__float_as_uint(G[u].w));
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k + u < n) body(G[u], g[u], q[u]);
    }
}

struct Two {
    float4 a, b;
};
struct Three {
    float4 a, b, c;
};
struct FiveF {
    float4 a, b, c;
    float d, e;
};

// Adds three per-thread values into parameter-gradient slots: a block sum first, then one FP64
// atomic per slot and block (every thread of the block calls it).
struct SumD {
    __device__ double operator()(double a, double b) const { return a + b; }
};
__device__ __forceinline__ void add_grads3(double* grads, int s0, int s1, int s2, double a, double b, double c) {
    a = block_reduce(a, SumD(), 0.0);
    b = block_reduce(b, SumD(), 0.0);
    c = block_reduce(c, SumD(), 0.0);
    if (threadIdx.x == 0) {
        atomicAdd(&grads[s0], a);
        atomicAdd(&grads[s1], b);
        atomicAdd(&grads[s2], c);
    }
}

__device__ __forceinline__ float3 f3(float4 a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float dotf(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }

// The adjoint's stiffness pass takes each list slot in one of two forms, as the forward check
// does: slot k uses the kept gradient G (PairLists::gv) when bit k % 4 of SLF_ADJ_KAPPA_GV_SLOTS
// is set, and otherwise gathers the neighbour's position and forms G = (x_i - x_j) g from its
// {index, g} entry.  The kept form streams more list bytes, the other gathers more; mixing them
// balances the two.
#ifndef SLF_ADJ_KAPPA_GV_SLOTS
#define SLF_ADJ_KAPPA_GV_SLOTS 0x7u
#endif
__device__ __forceinline__ bool kept_form(uint32_t k) { return (SLF_ADJ_KAPPA_GV_SLOTS >> (k & 3u)) & 1u; }

// body(G, gathered) for each of row's neighbours in list order, four at a time.
template <class Gather, class Body>
__device__ __forceinline__ void walk_gradients_mixed(const PairLists& l, uint32_t row, const float4* __restrict__ pos,
                                                     float3 xi, Gather&& gather, Body&& body) {
    uint32_t n = listed_count(l, row);
    if (n == 0) return;
    const float4* gb = l.gv + l.at(row, 0);
    const uint2* eb = l.e + l.at(row, 0);
    for (uint32_t k = 0; k < n; k += 4) {
        float4 G[4], q[4];
        uint32_t j[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t kk = k + u < n ? k + u : n - 1;
            if (kept_form(k + u)) {
                G[u] = SLF_LIST_LOAD(gb + size_t(kk) * 32u);
                j[u] = __float_as_uint(G[u].w);
            } else {
                const uint2 e = SLF_LIST_LOAD(eb + size_t(kk) * 32u);
                j[u] = e.x;
                G[u].w = __uint_as_float(e.y);  // g until the position arrives
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            q[u] = gather(j[u]);
            if (!kept_form(k + u)) {
                const float4 xj = __ldg(&pos[j[u]]);
                const float g = G[u].w;
                G[u] = make_float4((xi.x - xj.x) * g, (xi.y - xj.y) * g, (xi.z - xj.z) * g, 0.0f);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k + u < n) body(G[u], q[u]);
    }
}

// ---- terrain (terrain.rs) ------------------------------------------------------------------
// The trilinear distance is linear along each axis inside a cell: its second derivatives are
// zero on the diagonal and hxy, hxz, hyz off it.  hess_times(c, step, b) = H b.
__device__ __forceinline__ float3 hess_times(const TerrainCell& c, float step, float3 b) {
    float g00 = c.b00 - c.a00, g10 = c.b10 - c.a10, g01 = c.b01 - c.a01, g11 = c.b11 - c.a11;
    float v00 = c.a00 + g00 * c.fx, v10 = c.a10 + g10 * c.fx, v01 = c.a01 + g01 * c.fx, v11 = c.a11 + g11 * c.fx;
    float hxy = (g10 - g00) + ((g11 - g01) - (g10 - g00)) * c.fz;
    float hxz = (g01 + (g11 - g01) * c.fy) - (g00 + (g10 - g00) * c.fy);
    float hyz = (v11 - v01) - (v10 - v00);
    float s2 = 1.0f / (step * step);
    return make_float3((hxy * b.y + hxz * b.z) * s2, (hxy * b.x + hyz * b.z) * s2, (hxz * b.x + hyz * b.y) * s2);
}

// The adjoint of n = normalize_or(Y)(c): c-bar from n-bar (zero where the forward fell back to Y).
__device__ __forceinline__ float3 unit_adjoint(float3 c, float3 n, float3 nbar) {
    float len = sqrtf(c.x * c.x + c.y * c.y + c.z * c.z);
    if (!(isfinite(len) && len > 0.0f)) return make_float3(0.0f, 0.0f, 0.0f);
    return (nbar - n * dotf(n, nbar)) * (1.0f / len);
}

// The ground's slope at particle x (ground_near, terrain.rs:144-171, 305-310) is the sum over the
// sites whose solid share lies strictly inside (0, 1) of -change(x + o) w / spacing; returns
// (d slope / d x)^T b, the sites and their shares taken as the forward took them.
__device__ __forceinline__ float3 ground_slope_adjoint(const TerrainDev& T, float3 x, float3 b) {
    float3 out = make_float3(0.0f, 0.0f, 0.0f);
    const float half = __fdiv_rn(T.spacing, 2.0f);
    for (uint32_t r = 0; r < T.regions; ++r) {
        const TerrainRegion& t = T.region[r];
        float distance;
        float3 change;
        if (!terrain_read(T, t, x.x, x.y, x.z, distance, change)) continue;
        if (!(distance < T.reach)) continue;
        const float open = __fsub_rn(distance, half);
        for (uint32_t k = 0; k < T.sites; ++k) {
            if (__ldg(&T.far[k]) <= open) continue;
            const float4 o = __ldg(&T.site[k]);
            TerrainCell c;
            if (!terrain_cell(T, t, __fadd_rn(x.x, o.x), __fadd_rn(x.y, o.y), __fadd_rn(x.z, o.z), c)) continue;
            float there;
            float3 toward;
            terrain_values(c, t.step, there, toward);
            const float v = __fsub_rn(0.5f, __fdiv_rn(there, T.spacing));
            if (!(v > 0.0f && v < 1.0f)) continue;
            out = out - hess_times(c, t.step, b) * (o.w / T.spacing);
        }
    }
    return out;
}

// The ground's damping in the wall viscosity (step.rs:281-296): for each region holding x with
// v . n < 0, a -= n nu_w (v . n) weight(d) / rho.  Adds its adjoint for a-bar ai.
__device__ __forceinline__ void ground_damping_adjoint(const TerrainDev& T, float nuw, float3 x, float3 v, float rho,
                                                       float3 ai, float3& xbar, float3& vbar, float& rbar,
                                                       double& nuw_bar) {
    for (uint32_t r = 0; r < T.regions; ++r) {
        const TerrainRegion& t = T.region[r];
        TerrainCell c;
        if (!terrain_cell(T, t, x.x, x.y, x.z, c)) continue;
        float d;
        float3 ch;
        terrain_values(c, t.step, d, ch);
        const float3 n = normalize_or_up(ch);
        const float into = dot3(v.x, v.y, v.z, n.x, n.y, n.z);
        if (!(into < 0.0f)) continue;
        float wslope;
        const float weight = ground_damping(T, d, &wslope);
        const float cc = nuw * into * weight / rho;
        const float cbar = -dotf(ai, n);  // L = -cc (a-bar . n)
        const float intobar = cbar * nuw * weight / rho;
        rbar += -cbar * cc / rho;
        nuw_bar += (double)(cbar * into * weight / rho);
        vbar = vbar + n * intobar;
        const float3 nbar = ai * (-cc) + v * intobar;
        const float dbar = cbar * nuw * into / rho * wslope;
        xbar = xbar + ch * dbar + hess_times(c, t.step, unit_adjoint(ch, n, nbar));
    }
}

// The body points' push (couple.rs:375-416, mover_pairs): for each point within reach of x,
// a -= G (M + D) with G = m o g(|o|), o = x - point, and the damping D = -k tau / ((|o|^2 + eps)
// rho) where tau = (v - u) . o < 0 (u: the point's velocity).  Adds the adjoint for a-bar ai into
// x-bar, v-bar, rho-bar, M-bar (the mirrored pressure) and k-bar; the points' motion is given.
__device__ __forceinline__ void mover_adjoint(const Params& p, const MoverDev& B, float k, float3 xi, float3 vi,
                                              float rho, float mirrored, float3 ai, float3& xbar, float3& vbar,
                                              float& rbar, float& mbar, double& kbar) {
    const int3 cell = cell_of(p, xi.x, xi.y, xi.z);
    each_near(p, B.grid, B.pos, cell, xi.x, xi.y, xi.z, [&](uint32_t j, float4 q) {
        const float3 o = make_float3(xi.x - q.x, xi.y - q.y, xi.z - q.z);
        const float d2 = dotf(o, o), inv = inv_length(d2);
        if (inv == 0.0f) return;  // coincident: no gradient, and tau = 0 takes no damping
        float g, gp;
        grad_factor(p, d2 * inv, g, gp);
        const float3 u = vi - f3(__ldg(&B.vel[j]));
        const float tau = dotf(u, o);
        const bool act = tau < 0.0f;
        const float e2 = d2 + p.soften;
        const float D = act ? -k * tau / (e2 * rho) : 0.0f;
        const float A = dotf(ai, o);
        const float h = -p.mass * g * A;  // dL/dM = dL/dD
        mbar += h;
        xbar = xbar + (ai * g + o * (A * gp * inv)) * (-p.mass * (mirrored + D));
        if (act) {
            const float dtau = -k / (e2 * rho);  // dD/dtau
            xbar = xbar + u * (h * dtau) + o * (h * (-D / e2) * 2.0f);
            vbar = vbar + o * (h * dtau);
            rbar += h * (-D / rho);
            kbar += (double)(h * (-tau / (e2 * rho)));
        }
    });
}

// terrain_contact (terrain.rs:314-333) backwards: (ybar, vbar) after every region's contact ->
// before the first, the state before it (y0, v0) as the forward had it.  Each region's own state
// is found by running the regions before it again.
__device__ __forceinline__ void contact_adjoint(const TerrainDev& T, float rest, float3 y0, float4 v0, float3& ybar,
                                                float3& vbar) {
    for (uint32_t r = T.regions; r-- > 0;) {
        float3 y = y0;
        float4 v = v0;
        bool under = false;
        for (uint32_t q = 0; q < r; ++q) contact_region(T, T.region[q], rest, y.x, y.y, y.z, v, under);
        const TerrainRegion& t = T.region[r];
        TerrainCell c;
        if (!terrain_cell(T, t, y.x, y.y, y.z, c)) continue;
        float d;
        float3 ch;
        terrain_values(c, t.step, d, ch);
        if (!(d < rest)) continue;
        const float3 n = normalize_or_up(ch);
        const float into = dot3(v.x, v.y, v.z, n.x, n.y, n.z);
        // y' = y + n (rest - d); v' = v - n (v . n) when v . n < 0
        float3 nbar = ybar * (rest - d);
        const float dbar = -dotf(n, ybar);
        if (into < 0.0f) {
            const float nv = dotf(n, vbar);
            nbar = nbar - (vbar * into + f3(v) * nv);
            vbar = vbar - n * nv;
        }
        ybar = ybar + ch * dbar + hess_times(c, t.step, unit_adjoint(ch, n, nbar));
    }
}

// ---- advance and velocity update (step.rs:212-222, 305-339) ---------------------------------
// y = x + v' dt is clamped per component; a clamped component passes no adjoint to y and zeroes
// v'.  v' = v + a dt.  Gravity's gradient is the sum of a-bar.
// Terrain contact, after the clamp, goes back first (contact_adjoint): pos holds the substep's
// sorted positions, from which the forward's position before contact is formed again.
__global__ void k_adj_advance(Params p, const StepConsts* __restrict__ sc, const float4* __restrict__ vel_pre,
                              const float4* __restrict__ xo, const float4* __restrict__ vo,
                              float4* __restrict__ ab, float4* __restrict__ xb, float4* __restrict__ vb,
                              double* __restrict__ grads, const float4* __restrict__ pos, TerrainDev T) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    if (i < p.n) {
        const float dt = sc->dt;
        const float4 pre = vel_pre[i];
        uint32_t flags = __float_as_uint(pre.w);
        float4 x = xo[i], v = vo[i];
        if (T.regions) {
            // advance_one's position and velocity before contact: x + v' dt, clamped
            const float4 a = pos[i];
            float3 y = make_float3(__fadd_rn(a.x, __fmul_rn(pre.x, dt)), __fadd_rn(a.y, __fmul_rn(pre.y, dt)),
                                   __fadd_rn(a.z, __fmul_rn(pre.z, dt)));
            float4 w = make_float4(pre.x, pre.y, pre.z, 0.0f);
            if (p.has_bounds) {
                y = make_float3(fminf(fmaxf(y.x, p.low_in.x), p.high_in.x), fminf(fmaxf(y.y, p.low_in.y), p.high_in.y),
                                fminf(fmaxf(y.z, p.low_in.z), p.high_in.z));
                if (flags & 1u) w.x = 0.0f;
                if (flags & 2u) w.y = 0.0f;
                if (flags & 4u) w.z = 0.0f;
            }
            float3 ybar = f3(x), wbar = f3(v);
            contact_adjoint(T, __fdiv_rn(p.spacing, 2.0f), y, w, ybar, wbar);
            x = make_float4(ybar.x, ybar.y, ybar.z, 0.0f);
            v = make_float4(wbar.x, wbar.y, wbar.z, 0.0f);
        }
        float yx = flags & 1u ? 0.0f : x.x, yy = flags & 2u ? 0.0f : x.y, yz = flags & 4u ? 0.0f : x.z;
        float wx = (flags & 1u ? 0.0f : v.x) + yx * dt;
        float wy = (flags & 2u ? 0.0f : v.y) + yy * dt;
        float wz = (flags & 4u ? 0.0f : v.z) + yz * dt;
        ab[i] = make_float4(wx * dt, wy * dt, wz * dt, 0.0f);
        xb[i] = make_float4(yx, yy, yz, 0.0f);
        vb[i] = make_float4(wx, wy, wz, 0.0f);
        gx = wx * dt;
        gy = wy * dt;
        gz = wz * dt;
    }
    // gravity: a_i gets g, so g-bar = sum of a-bar
    add_grads3(grads, kGradGravity, kGradGravity + 1, kGradGravity + 2, gx, gy, gz);
}

// ---- forces (step.rs:173-211), wall viscosity (step.rs:262-301), Tait pressure (step.rs:147-172)
// PRESSURE = false: the DFSPH viscosity pass (dfsph.rs:90-99), the same pairs without pressure,
// so the pressure records are neither gathered nor differentiated
// TERRAIN: the ground's terms and the body points' as well (WCSPH worlds with terrain regions or
// coupled bodies)
template <bool PRESSURE, bool TERRAIN = false>
__global__ void __launch_bounds__(kBlock) k_adj_force(Params p, const StepConsts* __restrict__ sc, PairLists fl,
                                                      PairLists wl, int form, const float4* __restrict__ pos,
                                                      const float4* __restrict__ vel, const float* __restrict__ rho,
                                                      const float* __restrict__ press,
                                                      const float* __restrict__ scaled,
                                                      const float4* __restrict__ walls,
                                                      const float4* __restrict__ ab, float4* __restrict__ xb,
                                                      float4* __restrict__ vb, float* __restrict__ rb,
                                                      double* __restrict__ grads, int add_rho, TerrainDev T,
                                                      const float4* __restrict__ slope, MoverDev bodies) {
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = row < p.n ? fl.particle(row) : row;  // row of the walk order, its particle
    double nu_bar = 0.0, nuw_bar = 0.0, b_bar = 0.0;
    if (i < p.n) {
        const float nu = sc->viscosity, nuw = sc->wall_viscosity, m = p.mass;
        float3 xi = f3(pos[i]), vi = f3(vel[i]), ai = f3(ab[i]);
        float rho_i = rho[i], p_i = PRESSURE ? press[i] : 0.0f, s_i = PRESSURE ? scaled[i] : 0.0f;
        float3 xbar = make_float3(0, 0, 0), vbar = make_float3(0, 0, 0);
        float sbar = 0.0f, pbar = 0.0f, rbar = 0.0f;

        // fluid pairs: L = (a_i-bar - a_j-bar) . T(r, u, S, R)
        walk4<FiveF>(fl, form, row,
                     [&](uint32_t j) {
                         return FiveF{__ldg(&pos[j]), __ldg(&vel[j]), __ldg(&ab[j]), __ldg(&rho[j]),
                                      PRESSURE ? __ldg(&scaled[j]) : 0.0f};
                     },
                     [&](uint32_t, const FiveF& q, uint32_t e) {
            float3 r = pair_off(p, form, xi, q.a, e);
            float d2 = dotf(r, r), inv = inv_length(d2);
            if (inv == 0.0f) return;
            float g, gp;
            grad_factor(p, d2 * inv, g, gp);
            float3 u = vi - f3(q.b);
            float3 w = ai - f3(q.c);
            float R = rho_i + q.d;
            float S = PRESSURE ? s_i + q.e : 0.0f;
            // EXACT lists: the forward's own dot product decides whether the pair approaches
            float ur = form == kFormExact ? dot3(u.x, u.y, u.z, r.x, r.y, r.z) : dotf(u, r);
            bool act = ur < 0.0f;
            float t = act ? ur : 0.0f;
            float den = (d2 + p.soften) * R;
            float Pi = -nu * t * 2.0f / den;
            float G = dotf(w, r);
            float P = -m * g * G;  // dL/dPi and dL/dS
            float dPi_dt = -2.0f * nu / den;
            float dPi_dd2 = -Pi / (d2 + p.soften);
            float c1 = -m * (S + Pi);
            float3 dr = w * (c1 * g) + r * (c1 * G * gp * inv + P * dPi_dd2 * 2.0f);
            if (act) dr = dr + u * (P * dPi_dt);
            xbar = xbar + dr;
            if (act) vbar = vbar + r * (P * dPi_dt);
            rbar += P * (-Pi / R);
            if (PRESSURE) sbar += P;
            // viscosity enters a_i's own term: a_i-bar . dT/dnu
            nu_bar += (double)(2.0f * m * g * t * dotf(ai, r) / den);
        });

        // walls: pressure mirrored onto the wall (step.rs:197-202)
        uint32_t nw = listed_count(wl, row);
        float M = s_i + p_i * p.inv_rest_sq;
        float3 A = make_float3(0, 0, 0);  // sum of -grad W over walls, for the wall normal
        // EXACT lists: the same sum as the forward forms it (the entries' g, each operation on its
        // own), so that the normal's branches below are the forward's
        float3 Ae = make_float3(0, 0, 0);
        for (uint32_t k = 0; k < nw; ++k) {
            uint32_t e = listed_raw(wl, form, row, k), j = entry_index(e, form);
            float3 r = pair_off(p, form, xi, __ldg(&walls[j]), e);
            if (form == kFormExact) {
                const float ge = __uint_as_float(SLF_LIST_LOAD(&wl.e[wl.at(row, k)]).y);
                Ae = make_float3(__fadd_rn(Ae.x, -__fmul_rn(r.x, ge)), __fadd_rn(Ae.y, -__fmul_rn(r.y, ge)),
                                 __fadd_rn(Ae.z, -__fmul_rn(r.z, ge)));
            }
            float d2 = dotf(r, r), inv = inv_length(d2);
            if (inv == 0.0f) continue;
            float g, gp;
            grad_factor(p, d2 * inv, g, gp);
            if (PRESSURE) {
                float ar = dotf(ai, r);
                float mb = -m * g * ar;
                sbar += mb;
                pbar += mb * p.inv_rest_sq;
                xbar = xbar + (ai * g + r * (ar * gp * inv)) * (-m * M);
            }
            A = A - r * g;
        }

        // wall viscosity (step.rs:262-301): n = A / |A|, I = n min(v.n, 0), and per wall with
        // tau = I.r < 0: D = -nu_w tau / ((|r|^2 + eps) rho), push -= r g m D
        const bool exact = form == kFormExact;
        float alen = exact ? __fsqrt_rn(dot3(Ae.x, Ae.y, Ae.z, Ae.x, Ae.y, Ae.z)) : sqrtf(dotf(A, A));
        if (nw > 0 && alen > 0.0f && isfinite(alen)) {
            // EXACT lists: normal, v.n and each tau as the forward rounds them (wall_viscous)
            float3 nrm = exact ? make_float3(__fdiv_rn(Ae.x, alen), __fdiv_rn(Ae.y, alen), __fdiv_rn(Ae.z, alen))
                               : A * (1.0f / alen);
            float vn = exact ? dot3(vi.x, vi.y, vi.z, nrm.x, nrm.y, nrm.z) : dotf(vi, nrm);
            float kk = fminf(vn, 0.0f);
            float3 I = exact ? make_float3(__fmul_rn(nrm.x, kk), __fmul_rn(nrm.y, kk), __fmul_rn(nrm.z, kk)) : nrm * kk;
            float3 Ibar = make_float3(0, 0, 0);
            for (uint32_t k = 0; k < nw; ++k) {
                uint32_t e = listed_raw(wl, form, row, k), j = entry_index(e, form);
                float3 r = pair_off(p, form, xi, __ldg(&walls[j]), e);
                float tau = exact ? dot3(I.x, I.y, I.z, r.x, r.y, r.z) : dotf(I, r);
                if (!(tau < 0.0f)) continue;
                float d2 = dotf(r, r);
                float d = sqrtf(d2);
                float g, gp;
                grad_factor(p, d, g, gp);
                float e2 = d2 + p.soften;
                float D = -nuw * tau / (e2 * rho_i);
                float ar = dotf(ai, r);
                float h = -m * g * ar;  // L = sum D h
                float tb = h * (-nuw / (e2 * rho_i));
                rbar += -D * h / rho_i;
                nuw_bar += (double)(-tau / (e2 * rho_i) * h);
                // through h(r), through |r|^2 in D, through tau = I.r
                float3 dh = (ai * g + r * (ar * gp / d)) * (-m);
                xbar = xbar + dh * D + r * (h * (-D / e2) * 2.0f) + I * tb;
                Ibar = Ibar + r * tb;
            }
            // I = n k, k = min(v.n, 0)
            float3 nbar = Ibar * kk;
            if (vn < 0.0f) {
                float kbar = dotf(Ibar, nrm);
                vbar = vbar + nrm * kbar;
                nbar = nbar + vi * kbar;
            }
            // n = A / |A|
            float3 Abar = (nbar - nrm * dotf(nrm, nbar)) * (1.0f / alen);
            // A = sum -r g
            for (uint32_t k = 0; k < nw; ++k) {
                uint32_t e = listed_raw(wl, form, row, k), j = entry_index(e, form);
                float3 r = pair_off(p, form, xi, __ldg(&walls[j]), e);
                float d = sqrtf(dotf(r, r));
                if (d <= 0.0f) continue;
                float g, gp;
                grad_factor(p, d, g, gp);
                xbar = xbar - (Abar * g + r * (dotf(Abar, r) * gp / d));
            }
        }

        // terrain (WCSPH): the ground's push with the particle's own pressure (step.rs:203-205),
        // a -= slope M, and its damping in the wall viscosity
        if (PRESSURE && TERRAIN) {
            if (slope) {
                const float3 sl = f3(slope[i]);
                const float as = dotf(ai, sl);
                sbar -= as;
                pbar -= as * p.inv_rest_sq;
                xbar = xbar + ground_slope_adjoint(T, xi, ai * (-M));
            }
            ground_damping_adjoint(T, nuw, xi, vi, rho_i, ai, xbar, vbar, rbar, nuw_bar);
            if (bodies.count) {
                // the mover damping has the wall viscosity's form (couple.rs:375-416): its gradient
                // joins that slot
                float mbar = 0.0f;
                mover_adjoint(p, bodies, sc->mover_damping, xi, vi, rho_i, M, ai, xbar, vbar, rbar, mbar, nuw_bar);
                sbar += mbar;
                pbar += mbar * p.inv_rest_sq;
            }
        }

        // s = p / rho^2 and the Tait equation of state
        if (PRESSURE) {
            float ptot = pbar + sbar / (rho_i * rho_i);
            rbar += sbar * (-2.0f * p_i / (rho_i * rho_i * rho_i));
            float raw = rho_i * p.inv_rest;
            float ratio = fminf(raw, 1.1f);
            float r2 = ratio * ratio, r3 = r2 * ratio, r6 = r3 * r3;
            if (p_i > 0.0f) {
                b_bar = (double)(ptot * (r6 * ratio - 1.0f));
                if (raw < 1.1f) rbar += ptot * p.stiffness * 7.0f * r6 * p.inv_rest;
            }
        }
        float4 x0 = xb[i], v0 = vb[i];
        xb[i] = make_float4(x0.x + xbar.x, x0.y + xbar.y, x0.z + xbar.z, 0.0f);
        vb[i] = make_float4(v0.x + vbar.x, v0.y + vbar.y, v0.z + vbar.z, 0.0f);
        rb[i] = add_rho ? rb[i] + rbar : rbar;
    }
    add_grads3(grads, kGradViscosity, kGradWallViscosity, kGradStiffness, nu_bar, nuw_bar, b_bar);
}

// ---- the same two adjoints a warp a row, for scenes too small to fill the GPU a thread a row ----
// Each lane takes every 32nd entry of the row's lists; partial sums meet in butterfly sums, which
// leave every lane with the same bits (each level adds x + y on one lane and y + x on its partner),
// so the lanes agree on the wall normal they all form.  Run to run the sums are deterministic.
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float3 warp_sum3(float3 v) { return make_float3(warp_sum(v.x), warp_sum(v.y), warp_sum(v.z)); }

constexpr uint32_t kAdjWarpMax = 262144u;  // rows a warp each up to this many particles

// k_adj_force (WCSPH forces, wall viscosity, Tait pressure) a warp a row; no terrain.
__global__ void __launch_bounds__(kBlock) k_adj_force_warp(Params p, const StepConsts* __restrict__ sc, PairLists fl,
                                                           PairLists wl, int form, const float4* __restrict__ pos,
                                                           const float4* __restrict__ vel, const float* __restrict__ rho,
                                                           const float* __restrict__ press,
                                                           const float* __restrict__ scaled,
                                                           const float4* __restrict__ walls,
                                                           const float4* __restrict__ ab, float4* __restrict__ xb,
                                                           float4* __restrict__ vb, float* __restrict__ rb,
                                                           double* __restrict__ grads) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
    double nu_bar = 0.0, nuw_bar = 0.0, b_bar = 0.0;
    if (row < p.n) {
        const uint32_t i = fl.particle(row);
        const float nu = sc->viscosity, nuw = sc->wall_viscosity, m = p.mass;
        const float3 xi = f3(pos[i]), vi = f3(vel[i]), ai = f3(ab[i]);
        const float rho_i = rho[i], p_i = press[i], s_i = scaled[i];
        float3 xbar = make_float3(0, 0, 0), vbar = make_float3(0, 0, 0);
        float sbar = 0.0f, pbar = 0.0f, rbar = 0.0f;

        // fluid pairs: L = (a_i-bar - a_j-bar) . T(r, u, S, R)
        const uint32_t nf = listed_count(fl, row);
        for (uint32_t k = lane; k < nf; k += 32u) {
            const uint32_t e = listed_raw(fl, form, row, k), j = entry_index(e, form);
            const float4 qa = __ldg(&pos[j]), qv = __ldg(&vel[j]), qb = __ldg(&ab[j]);
            const float qr = __ldg(&rho[j]), qs = __ldg(&scaled[j]);
            float3 r = pair_off(p, form, xi, qa, e);
            float d2 = dotf(r, r), inv = inv_length(d2);
            if (inv == 0.0f) continue;
            float g, gp;
            grad_factor(p, d2 * inv, g, gp);
            float3 u = vi - f3(qv);
            float3 w = ai - f3(qb);
            float R = rho_i + qr;
            float S = s_i + qs;
            // EXACT lists: the forward's own dot product decides whether the pair approaches
            float ur = form == kFormExact ? dot3(u.x, u.y, u.z, r.x, r.y, r.z) : dotf(u, r);
            bool act = ur < 0.0f;
            float t = act ? ur : 0.0f;
            float den = (d2 + p.soften) * R;
            float Pi = -nu * t * 2.0f / den;
            float G = dotf(w, r);
            float P = -m * g * G;
            float dPi_dt = -2.0f * nu / den;
            float dPi_dd2 = -Pi / (d2 + p.soften);
            float c1 = -m * (S + Pi);
            float3 dr = w * (c1 * g) + r * (c1 * G * gp * inv + P * dPi_dd2 * 2.0f);
            if (act) dr = dr + u * (P * dPi_dt);
            xbar = xbar + dr;
            if (act) vbar = vbar + r * (P * dPi_dt);
            rbar += P * (-Pi / R);
            sbar += P;
            nu_bar += (double)(2.0f * m * g * t * dotf(ai, r) / den);
        }

        // walls: pressure mirrored onto the wall, and the wall normal's sum
        const uint32_t nw = listed_count(wl, row);
        const float M = s_i + p_i * p.inv_rest_sq;
        float3 A = make_float3(0, 0, 0);
        for (uint32_t k = lane; k < nw; k += 32u) {
            const uint32_t e = listed_raw(wl, form, row, k), j = entry_index(e, form);
            float3 r = pair_off(p, form, xi, __ldg(&walls[j]), e);
            float d2 = dotf(r, r), inv = inv_length(d2);
            if (inv == 0.0f) continue;
            float g, gp;
            grad_factor(p, d2 * inv, g, gp);
            float ar = dotf(ai, r);
            float mb = -m * g * ar;
            sbar += mb;
            pbar += mb * p.inv_rest_sq;
            xbar = xbar + (ai * g + r * (ar * gp * inv)) * (-m * M);
            A = A - r * g;
        }
        A = warp_sum3(A);

        // wall viscosity (every lane holds the same A, so the same normal and branch)
        float alen = sqrtf(dotf(A, A));
        if (nw > 0 && alen > 0.0f && isfinite(alen)) {
            float3 nrm = A * (1.0f / alen);
            float vn = dotf(vi, nrm);
            float kk = fminf(vn, 0.0f);
            float3 I = nrm * kk;
            float3 Ibar = make_float3(0, 0, 0);
            for (uint32_t k = lane; k < nw; k += 32u) {
                const uint32_t e = listed_raw(wl, form, row, k), j = entry_index(e, form);
                float3 r = pair_off(p, form, xi, __ldg(&walls[j]), e);
                float tau = dotf(I, r);
                if (!(tau < 0.0f)) continue;
                float d2 = dotf(r, r);
                float d = sqrtf(d2);
                float g, gp;
                grad_factor(p, d, g, gp);
                float e2 = d2 + p.soften;
                float D = -nuw * tau / (e2 * rho_i);
                float ar = dotf(ai, r);
                float h = -m * g * ar;
                float tb = h * (-nuw / (e2 * rho_i));
                rbar += -D * h / rho_i;
                nuw_bar += (double)(-tau / (e2 * rho_i) * h);
                float3 dh = (ai * g + r * (ar * gp / d)) * (-m);
                xbar = xbar + dh * D + r * (h * (-D / e2) * 2.0f) + I * tb;
                Ibar = Ibar + r * tb;
            }
            Ibar = warp_sum3(Ibar);
            float3 nbar = Ibar * kk;
            if (vn < 0.0f) {
                float kbar = dotf(Ibar, nrm);
                if (lane == 0) vbar = vbar + nrm * kbar;
                nbar = nbar + vi * kbar;
            }
            float3 Abar = (nbar - nrm * dotf(nrm, nbar)) * (1.0f / alen);
            for (uint32_t k = lane; k < nw; k += 32u) {
                const uint32_t e = listed_raw(wl, form, row, k), j = entry_index(e, form);
                float3 r = pair_off(p, form, xi, __ldg(&walls[j]), e);
                float d = sqrtf(dotf(r, r));
                if (d <= 0.0f) continue;
                float g, gp;
                grad_factor(p, d, g, gp);
                xbar = xbar - (Abar * g + r * (dotf(Abar, r) * gp / d));
            }
        }

        xbar = warp_sum3(xbar);
        vbar = warp_sum3(vbar);
        sbar = warp_sum(sbar);
        pbar = warp_sum(pbar);
        rbar = warp_sum(rbar);
        if (lane == 0) {
            // s = p / rho^2 and the Tait equation of state
            float ptot = pbar + sbar / (rho_i * rho_i);
            rbar += sbar * (-2.0f * p_i / (rho_i * rho_i * rho_i));
            float raw = rho_i * p.inv_rest;
            float ratio = fminf(raw, 1.1f);
            float r2 = ratio * ratio, r3 = r2 * ratio, r6 = r3 * r3;
            if (p_i > 0.0f) {
                b_bar = (double)(ptot * (r6 * ratio - 1.0f));
                if (raw < 1.1f) rbar += ptot * p.stiffness * 7.0f * r6 * p.inv_rest;
            }
            float4 x0 = xb[i], v0 = vb[i];
            xb[i] = make_float4(x0.x + xbar.x, x0.y + xbar.y, x0.z + xbar.z, 0.0f);
            vb[i] = make_float4(v0.x + vbar.x, v0.y + vbar.y, v0.z + vbar.z, 0.0f);
            rb[i] = rbar;
        }
    }
    add_grads3(grads, kGradViscosity, kGradWallViscosity, kGradStiffness, nu_bar, nuw_bar, b_bar);
}

// k_adj_density a warp a row.
__global__ void __launch_bounds__(kBlock) k_adj_density_warp(Params p, PairLists fl, PairLists wl, int form,
                                                             const float4* __restrict__ pos,
                                                             const float4* __restrict__ walls,
                                                             const float* __restrict__ rb, float4* __restrict__ xb) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
    if (row >= p.n) return;
    const uint32_t i = fl.particle(row);
    const float3 xi = f3(pos[i]);
    const float rbi = rb[i];
    float3 xbar = make_float3(0, 0, 0);
    const uint32_t nf = listed_count(fl, row);
    for (uint32_t k = lane; k < nf; k += 32u) {
        const uint32_t e = listed_raw(fl, form, row, k), j = entry_index(e, form);
        const float4 q = __ldg(&pos[j]);
        float3 r = pair_off(p, form, xi, q, e);
        float d = sqrtf(dotf(r, r));
        if (d <= 0.0f) continue;
        float g, gp;
        grad_factor(p, d, g, gp);
        xbar = xbar + r * (g * p.mass * (rbi + __ldg(&rb[j])));
    }
    const uint32_t nw = listed_count(wl, row);
    for (uint32_t k = lane; k < nw; k += 32u) {
        const uint32_t e = listed_raw(wl, form, row, k), j = entry_index(e, form);
        float3 r = pair_off(p, form, xi, __ldg(&walls[j]), e);
        float d = sqrtf(dotf(r, r));
        if (d <= 0.0f) continue;
        float g, gp;
        grad_factor(p, d, g, gp);
        xbar = xbar + r * (g * p.mass * rbi);
    }
    xbar = warp_sum3(xbar);
    if (lane == 0) {
        float4 x0 = xb[i];
        xb[i] = make_float4(x0.x + xbar.x, x0.y + xbar.y, x0.z + xbar.z, 0.0f);
    }
}

// ---- densities (mod.rs:621-675): rho_i = m (sum_j W(r_ij) + sum_w W(r_iw)) ---------------------
// slope (optional): the ground's density gradient of each particle, from the density pass (the
// ground's part of rho, whose derivative it is)
__global__ void __launch_bounds__(kBlock) k_adj_density(Params p, PairLists fl, PairLists wl, int form,
                                                        const float4* __restrict__ pos,
                                                        const float4* __restrict__ walls,
                                                        const float* __restrict__ rb, float4* __restrict__ xb,
                                                        const float4* __restrict__ slope, MoverDev bodies) {
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = row < p.n ? fl.particle(row) : row;  // row of the walk order, its particle
    if (i >= p.n) return;
    float3 xi = f3(pos[i]);
    float rbi = rb[i];
    float3 xbar = make_float3(0, 0, 0);
    walk4<float4>(fl, form, row,
                  [&](uint32_t j) {
                      float4 q = __ldg(&pos[j]);
                      q.w = __ldg(&rb[j]);
                      return q;
                  },
                  [&](uint32_t, float4 q, uint32_t e) {
                      float3 r = pair_off(p, form, xi, q, e);
                      float d = sqrtf(dotf(r, r));
                      if (d <= 0.0f) return;
                      float g, gp;
                      grad_factor(p, d, g, gp);
                      xbar = xbar + r * (g * p.mass * (rbi + q.w));
                  });
    uint32_t nw = listed_count(wl, row);
    for (uint32_t k = 0; k < nw; ++k) {
        uint32_t e = listed_raw(wl, form, row, k), j = entry_index(e, form);
        float3 r = pair_off(p, form, xi, __ldg(&walls[j]), e);
        float d = sqrtf(dotf(r, r));
        if (d <= 0.0f) continue;
        float g, gp;
        grad_factor(p, d, g, gp);
        xbar = xbar + r * (g * p.mass * rbi);
    }
    if (slope) xbar = xbar + f3(slope[i]) * rbi;
    if (bodies.count) {  // the body points' kernel sum (mod.rs:648-656)
        const int3 cell = cell_of(p, xi.x, xi.y, xi.z);
        each_near(p, bodies.grid, bodies.pos, cell, xi.x, xi.y, xi.z, [&](uint32_t, float4 q) {
            const float3 o = make_float3(xi.x - q.x, xi.y - q.y, xi.z - q.z);
            const float d = sqrtf(dotf(o, o));
            if (d <= 0.0f) return;
            float g, gp;
            grad_factor(p, d, g, gp);
            xbar = xbar + o * (g * p.mass * rbi);
        });
    }
    float4 x0 = xb[i];
    xb[i] = make_float4(x0.x + xbar.x, x0.y + xbar.y, x0.z + xbar.z, 0.0f);
}

// ---- the sort (mod.rs:541-566): back to the order before it ------------------------------------
// (ib, ip: the warm starts' impulse adjoint, when the solves start warm)
__global__ void k_adj_unsort(uint32_t n, const uint32_t* __restrict__ dest, const float4* __restrict__ xb,
                             const float4* __restrict__ vb, float4* __restrict__ xp, float4* __restrict__ vp,
                             const float2* __restrict__ ib, float2* __restrict__ ip) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t f = dest[i];
    xp[i] = xb[f];
    vp[i] = vb[f];
    if (ib) ip[i] = ib[f];
}

// ---- DFSPH (dfsph.rs:79-275) --------------------------------------------------------------------
// Within a substep the solves are linear in the velocities apart from the clamps of the stiffness:
// push_apart (dfsph.rs:184-216) is the transpose of density_rate (dfsph.rs:166-181) up to -dt, so
// the adjoint of a push is a rate pass on the velocity adjoint, and the adjoint of a rate pass is
// a push pass on the rate adjoint.

// advance (step.rs:305-339): the clamp passes nothing through clamped components
__global__ void k_adj_advance_dfsph(Params p, const StepConsts* __restrict__ sc, const float4* __restrict__ vel_pre,
                                    const float4* __restrict__ xo, const float4* __restrict__ vo,
                                    float4* __restrict__ xb, float4* __restrict__ w) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const float dt = sc->dt;
    uint32_t flags = __float_as_uint(vel_pre[i].w);
    float4 x = xo[i], v = vo[i];
    float yx = flags & 1u ? 0.0f : x.x, yy = flags & 2u ? 0.0f : x.y, yz = flags & 4u ? 0.0f : x.z;
    xb[i] = make_float4(yx, yy, yz, 0.0f);
    w[i] = make_float4((flags & 1u ? 0.0f : v.x) + yx * dt, (flags & 2u ? 0.0f : v.y) + yy * dt,
                       (flags & 4u ? 0.0f : v.z) + yz * dt, 0.0f);
}

// density_rate (dfsph.rs:166-181) of the velocity adjoint w at row's particle i, without its mass:
// sum_j (w_i - w_j) . grad W_ij + sum_walls w_i . grad W_iw, over the substep's lists.
__device__ __forceinline__ float adjoint_rate(const Params& p, const PairLists& fl, const PairLists& wl, int form,
                                              const float4* __restrict__ pos, const float4* __restrict__ walls,
                                              const float4* __restrict__ w, uint32_t row, float3 xi, float3 wi) {
    float acc = 0.0f;
    if (fl.gv && wl.gv) {
        // the forward's kept gradients (EXACT DFSPH): rate(w) gathers only w of each neighbour
        walk_gradients_mixed(fl, row, pos, xi, [&](uint32_t j) { return __ldg(&w[j]); },
                             [&](float4 G, float4 wj) { acc += dotf(wi - f3(wj), f3(G)); });
        uint32_t nw = listed_count(wl, row);
        const float4* wg = wl.gv + wl.at(row, 0);
        for (uint32_t k = 0; k < nw; ++k) acc += dotf(wi, f3(SLF_LIST_LOAD(wg + size_t(k) * 32u)));
    } else {
        walk4<Two>(fl, form, row, [&](uint32_t j) { return Two{__ldg(&pos[j]), __ldg(&w[j])}; },
                   [&](uint32_t, const Two& q, uint32_t e) {
                       float3 r = pair_off(p, form, xi, q.a, e);
                       float d2 = dotf(r, r), inv = inv_length(d2);
                       if (inv == 0.0f) return;
                       float g, gp;
                       grad_factor(p, d2 * inv, g, gp);
                       acc += dotf(wi - f3(q.b), r) * g;
                   });
        uint32_t nw = listed_count(wl, row);
        for (uint32_t k = 0; k < nw; ++k) {
            uint32_t e = listed_raw(wl, form, row, k), j = entry_index(e, form);
            float3 r = pair_off(p, form, xi, __ldg(&walls[j]), e);
            float d2 = dotf(r, r), inv = inv_length(d2);
            if (inv == 0.0f) continue;
            float g, gp;
            grad_factor(p, d2 * inv, g, gp);
            acc += dotf(wi, r) * g;
        }
    }
    return acc;
}

// One iteration's stiffness, back from the velocity adjoint w after its push: kappa-bar = -dt
// rate(w); then through kappa = phi(rate) alpha (dfsph.rs:241-259).
// Writes kw = (w, kappa) and vr = (v, rate-bar) per particle: the three records k_adj_push
// gathers per neighbour (with the position).
template <int WHICH>
__device__ __forceinline__ void adj_kappa_row(Params p, const StepConsts* __restrict__ sc, PairLists fl,
                                                      PairLists wl, int form, const float4* __restrict__ pos,
                                                      const float4* __restrict__ walls,
                                                      const float4* __restrict__ w, const float* __restrict__ rate,
                                                      const float* __restrict__ alpha, const float* __restrict__ rho,
                                                      const float4* __restrict__ vel, float4* __restrict__ kw,
                                                      float4* __restrict__ vr, float* __restrict__ abar,
                                                      float* __restrict__ rb, const float2* __restrict__ appbar,
                                                      uint32_t row) {
    const uint32_t i = fl.particle(row);  // row of the walk order, its particle
    const float dt = sc->dt, m = p.mass;
    float3 xi = f3(pos[i]), wi = f3(w[i]);
    float kbar = -dt * m * adjoint_rate(p, fl, wl, form, pos, walls, w, row, xi, wi);
    // warm starts: the impulse the solve leaves sums each push's kappa dt (applied-bar of WHICH)
    if (appbar) kbar += dt * (WHICH == 1 ? appbar[i].y : appbar[i].x);
    float ri = rate[i], ai = alpha[i];
    float phi, dphi, dphi_rho = 0.0f;
    if (WHICH == 1) {
        // the forward's rounding, each operation on its own (no contraction): particles at rest
        // density sit within an ulp of the clamp, and the branch must be the forward's
        float over = __fsub_rn(__fadd_rn(rho[i], __fmul_rn(dt, ri)), p.rest);
        bool on = over > 0.0f;
        phi = on ? over / sc->dt_sq : 0.0f;
        dphi = on ? 1.0f / dt : 0.0f;
        dphi_rho = on ? 1.0f / sc->dt_sq : 0.0f;
    } else {
        bool on = fl.count[row] + wl.count[row] >= 20u && ri > 0.0f;
        phi = on ? ri / dt : 0.0f;
        dphi = on ? 1.0f / dt : 0.0f;
    }
    float4 v = vel[i];
    kw[i] = make_float4(wi.x, wi.y, wi.z, phi * ai);
    vr[i] = make_float4(v.x, v.y, v.z, kbar * ai * dphi);
    abar[i] += kbar * phi;
    if (WHICH == 1) rb[i] += kbar * ai * dphi_rho;
}

template <int WHICH>
__global__ void __launch_bounds__(kBlock) k_adj_kappa(Params p, const StepConsts* __restrict__ sc, PairLists fl,
                                                      PairLists wl, int form, const float4* __restrict__ pos,
                                                      const float4* __restrict__ walls,
                                                      const float4* __restrict__ w, const float* __restrict__ rate,
                                                      const float* __restrict__ alpha, const float* __restrict__ rho,
                                                      const float4* __restrict__ vel, float4* __restrict__ kw,
                                                      float4* __restrict__ vr, float* __restrict__ abar,
                                                      float* __restrict__ rb, const float2* __restrict__ appbar) {
    // rows a grid's width apart (one each when the grid covers them all)
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < p.n; row += gridDim.x * blockDim.x)
        adj_kappa_row<WHICH>(p, sc, fl, wl, form, pos, walls, w, rate, alpha, rho, vel, kw, vr, abar, rb, appbar,
                             row);
}

// The warm push of a solve (dfsph.rs's cold start replaced by one push at kappa_w = share applied /
// dt before the first check): kappa_w-bar from the velocity adjoint w after it, as the stiffness
// pass forms kappa-bar, plus dt applied-bar (the solve's impulse starts at kappa_w dt); the records
// k_adj_push then reads (rate-bar and velocities zero: the push moves only positions' adjoint), and
// applied-bar before the solve, kappa_w-bar share / dt, into component WHICH of appbar_out.
template <int WHICH>
__global__ void __launch_bounds__(kBlock) k_adj_warm(Params p, const StepConsts* __restrict__ sc, PairLists fl,
                                                     PairLists wl, int form, const float4* __restrict__ pos,
                                                     const float4* __restrict__ walls, const float4* __restrict__ w,
                                                     const float2* __restrict__ applied,
                                                     const float2* __restrict__ appbar, float share,
                                                     float4* __restrict__ kw, float4* __restrict__ vr,
                                                     float2* __restrict__ appbar_out) {
    const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= p.n) return;
    const uint32_t i = fl.particle(row);
    const float dt = sc->dt, m = p.mass;
    const float3 xi = f3(pos[i]), wi = f3(w[i]);
    float kbar = -dt * m * adjoint_rate(p, fl, wl, form, pos, walls, w, row, xi, wi);
    kbar += dt * (WHICH == 1 ? appbar[i].y : appbar[i].x);
    // the forward's kappa_w, rounded as k_warm_kappa rounds it
    const float kappa = __fdiv_rn(__fmul_rn(share, WHICH == 1 ? applied[i].y : applied[i].x), dt);
    kw[i] = make_float4(wi.x, wi.y, wi.z, kappa);
    vr[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    reinterpret_cast<float*>(appbar_out)[2 * size_t(i) + WHICH] = kbar * share / dt;
}

// The velocity adjoint before the iteration: w plus the rate pass's transpose (a push on the
// rate adjoint); and the positions' share of both passes, through grad W.
// four blocks a SM (64 registers)
// GV: the forward kept each pair's gradient (EXACT DFSPH), read in place of the position gather.
#ifndef SLF_ADJ_PUSH_GV_UNROLL
#define SLF_ADJ_PUSH_GV_UNROLL 2
#endif
#ifndef SLF_ADJ_PUSH_GV_BLOCKS
#define SLF_ADJ_PUSH_GV_BLOCKS 4
#endif
template <bool GV>
__device__ __forceinline__ void adj_push_row(Params p, const StepConsts* __restrict__ sc, PairLists fl,
                                                     PairLists wl, int form, const float4* __restrict__ pos,
                                                     const float4* __restrict__ walls, const float4* __restrict__ kw,
                                                     const float4* __restrict__ vr, float4* __restrict__ wout,
                                                     float4* __restrict__ xb, uint32_t row) {
    const uint32_t i = fl.particle(row);  // row of the walk order, its particle
    const float dt = sc->dt, m = p.mass;
    float4 own_w = kw[i], own_v = vr[i];
    float3 xi = f3(pos[i]), wi = f3(own_w), vi = f3(own_v);
    float ki = own_w.w, rbi = own_v.w;
    float3 vacc = make_float3(0, 0, 0), xacc = make_float3(0, 0, 0);
    if (GV) {
        // the forward's kept gradients (EXACT DFSPH): r = G / g and |r| = |G| / |g| from the
        // pair's entries, so only the two adjoint records of the neighbour are gathered
        walk_gradients_g<Two, SLF_ADJ_PUSH_GV_UNROLL>(fl, row, [&](uint32_t j) { return Two{__ldg(&kw[j]), __ldg(&vr[j])}; },
                              [&](float4 Gq, float g, const Two& q) {
                                  if (g == 0.0f) return;  // coincident: the pair adds nothing
                                  const float3 G = f3(Gq);
                                  const float ig = 1.0f / g;
                                  const float3 r = G * ig;
                                  float d2 = dotf(r, r), inv = inv_length(d2);
                                  if (inv == 0.0f) return;
                                  float gd, gp;
                                  grad_factor(p, d2 * inv, gd, gp);
                                  float rbj = q.b.w;
                                  vacc = vacc + G * (m * (rbi + rbj));
                                  float3 c = (wi - f3(q.a)) * (-dt * m * (ki + q.a.w)) + (vi - f3(q.b)) * (m * (rbi + rbj));
                                  xacc = xacc + c * g + r * (dotf(c, r) * gp * inv);
                              });
        uint32_t nw = listed_count(wl, row);
        const float4* wgb = wl.gv + wl.at(row, 0);
        for (uint32_t k = 0; k < nw; ++k) {
            const float g = __uint_as_float(SLF_LIST_LOAD(wl.e + wl.at(row, k)).y);
            if (g == 0.0f) continue;
            const float3 G = f3(SLF_LIST_LOAD(wgb + size_t(k) * 32u));
            const float3 r = G * (1.0f / g);
            float d2 = dotf(r, r), inv = inv_length(d2);
            if (inv == 0.0f) continue;
            float gd, gp;
            grad_factor(p, d2 * inv, gd, gp);
            vacc = vacc + G * (m * rbi);
            float3 c = wi * (-dt * m * ki) + vi * (m * rbi);
            xacc = xacc + c * g + r * (dotf(c, r) * gp * inv);
        }
        wout[i] = make_float4(wi.x + vacc.x, wi.y + vacc.y, wi.z + vacc.z, 0.0f);
        float4 x0 = xb[i];
        xb[i] = make_float4(x0.x + xacc.x, x0.y + xacc.y, x0.z + xacc.z, 0.0f);
        return;
    }
    walk4<Three, false>(fl, form, row,
                 [&](uint32_t j) { return Three{__ldg(&pos[j]), __ldg(&kw[j]), __ldg(&vr[j])}; },
                 [&](uint32_t, const Three& q, uint32_t e) {
                     float3 r = pair_off(p, form, xi, q.a, e);
                     float d2 = dotf(r, r), inv = inv_length(d2);
                     if (inv == 0.0f) return;
                     float g, gp;
                     grad_factor(p, d2 * inv, g, gp);
                     float rbj = q.c.w;
                     vacc = vacc + r * (g * m * (rbi + rbj));
                     // c . grad W(r) with c = -dt m (k_i + k_j)(w_i - w_j) + m (rb_i + rb_j)(v_i - v_j)
                     float3 c = (wi - f3(q.b)) * (-dt * m * (ki + q.b.w)) + (vi - f3(q.c)) * (m * (rbi + rbj));
                     xacc = xacc + c * g + r * (dotf(c, r) * gp * inv);
                 });
    uint32_t nw = listed_count(wl, row);
    for (uint32_t k = 0; k < nw; ++k) {
        uint32_t e = listed_raw(wl, form, row, k), j = entry_index(e, form);
        float3 r = pair_off(p, form, xi, __ldg(&walls[j]), e);
        float d2 = dotf(r, r), inv = inv_length(d2);
        if (inv == 0.0f) continue;
        float g, gp;
        grad_factor(p, d2 * inv, g, gp);
        vacc = vacc + r * (g * m * rbi);
        float3 c = wi * (-dt * m * ki) + vi * (m * rbi);
        xacc = xacc + c * g + r * (dotf(c, r) * gp * inv);
    }
    wout[i] = make_float4(wi.x + vacc.x, wi.y + vacc.y, wi.z + vacc.z, 0.0f);
    float4 x0 = xb[i];
    xb[i] = make_float4(x0.x + xacc.x, x0.y + xacc.y, x0.z + xacc.z, 0.0f);
}

template <bool GV>
__global__ void __launch_bounds__(kBlock, GV ? SLF_ADJ_PUSH_GV_BLOCKS : 4) k_adj_push(Params p, const StepConsts* __restrict__ sc, PairLists fl,
                                                     PairLists wl, int form, const float4* __restrict__ pos,
                                                     const float4* __restrict__ walls, const float4* __restrict__ kw,
                                                     const float4* __restrict__ vr, float4* __restrict__ wout,
                                                     float4* __restrict__ xb) {
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < p.n; row += gridDim.x * blockDim.x)
        adj_push_row<GV>(p, sc, fl, wl, form, pos, walls, kw, vr, wout, xb, row);
}

// viscosity + gravity (dfsph.rs:90-99): a-bar = dt w, gravity-bar = sum a-bar
__global__ void k_adj_scale(Params p, const StepConsts* __restrict__ sc, const float4* __restrict__ w,
                            float4* __restrict__ ab, double* __restrict__ grads) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    if (i < p.n) {
        float4 v = w[i];
        float dt = sc->dt;
        ab[i] = make_float4(v.x * dt, v.y * dt, v.z * dt, 0.0f);
        gx = v.x * dt;
        gy = v.y * dt;
        gz = v.z * dt;
    }
    add_grads3(grads, kGradGravity, kGradGravity + 1, kGradGravity + 2, gx, gy, gz);
}

// factors (dfsph.rs:138-163): alpha = 1 / T, T = |G|^2 + sum_j |m grad W_ij|^2,
// G = sum_j m grad W_ij + sum_w m grad W_iw.  First G and T-bar = -alpha-bar alpha^2 per particle.
__global__ void __launch_bounds__(kBlock) k_adj_alpha_prep(Params p, PairLists fl, PairLists wl, int form,
                                                           const float4* __restrict__ pos,
                                                           const float4* __restrict__ walls,
                                                           const float* __restrict__ alpha,
                                                           const float* __restrict__ abar, float4* __restrict__ gt) {
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = row < p.n ? fl.particle(row) : row;  // row of the walk order, its particle
    if (i >= p.n) return;
    float3 xi = f3(pos[i]);
    float3 G = make_float3(0, 0, 0);
    walk4<float4>(fl, form, row, [&](uint32_t j) { return __ldg(&pos[j]); }, [&](uint32_t, float4 q, uint32_t e) {
        float3 r = pair_off(p, form, xi, q, e);
        float d = sqrtf(dotf(r, r));
        if (d <= 0.0f) return;
        float g, gp;
        grad_factor(p, d, g, gp);
        G = G + r * (g * p.mass);
    });
    uint32_t nw = listed_count(wl, row);
    for (uint32_t k = 0; k < nw; ++k) {
        uint32_t e = listed_raw(wl, form, row, k), j = entry_index(e, form);
        float3 r = pair_off(p, form, xi, __ldg(&walls[j]), e);
        float d = sqrtf(dotf(r, r));
        if (d <= 0.0f) continue;
        float g, gp;
        grad_factor(p, d, g, gp);
        G = G + r * (g * p.mass);
    }
    float a = alpha[i];
    gt[i] = make_float4(G.x, G.y, G.z, -abar[i] * a * a);
}

__global__ void __launch_bounds__(kBlock) k_adj_alpha(Params p, PairLists fl, PairLists wl, int form,
                                                      const float4* __restrict__ pos,
                                                      const float4* __restrict__ walls,
                                                      const float4* __restrict__ gt, float4* __restrict__ xb) {
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = row < p.n ? fl.particle(row) : row;  // row of the walk order, its particle
    if (i >= p.n) return;
    const float m = p.mass;
    float3 xi = f3(pos[i]);
    float4 own = gt[i];
    float3 Gi = f3(own);
    float tbi = own.w;
    float3 xacc = make_float3(0, 0, 0);
    walk4<Two>(fl, form, row, [&](uint32_t j) { return Two{__ldg(&pos[j]), __ldg(&gt[j])}; },
               [&](uint32_t, const Two& q, uint32_t e) {
                   float3 r = pair_off(p, form, xi, q.a, e);
                   float d = sqrtf(dotf(r, r));
                   if (d <= 0.0f) return;
                   float g, gp;
                   grad_factor(p, d, g, gp);
                   float3 gw = r * (g * m);
                   float4 oj = q.b;
                   float3 c = (Gi + gw) * (2.0f * m * tbi) - (f3(oj) - gw) * (2.0f * m * oj.w);
                   xacc = xacc + c * g + r * (dotf(c, r) * gp / d);
               });
    uint32_t nw = listed_count(wl, row);
    for (uint32_t k = 0; k < nw; ++k) {
        uint32_t e = listed_raw(wl, form, row, k), j = entry_index(e, form);
        float3 r = pair_off(p, form, xi, __ldg(&walls[j]), e);
        float d = sqrtf(dotf(r, r));
        if (d <= 0.0f) continue;
        float g, gp;
        grad_factor(p, d, g, gp);
        float3 c = Gi * (2.0f * m * tbi);
        xacc = xacc + c * g + r * (dotf(c, r) * gp / d);
    }
    float4 x0 = xb[i];
    xb[i] = make_float4(x0.x + xacc.x, x0.y + xacc.y, x0.z + xacc.z, 0.0f);
}

static inline uint32_t adj_blocks(uint32_t n) {
    note_launch();
    return (n + kBlock - 1) / kBlock;
}

// The adjoint's stiffness passes on grids no larger than the SMs hold at once, each block striding
// over rows (k_adj_kappa<0>, <1>; 0: not looked up yet): 127 -> 123 us at 1M.  The adjoint push
// keeps a block a 256 rows (on the resident grid: 205 -> 218 us).
static std::atomic<uint32_t> g_adj_resident[2] = {0, 0};

void prepare_adjoint_grids() {
    if (g_adj_resident[1].load()) return;
    int dev = 0, sms = 0, per[2] = {0, 0};
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[0], k_adj_kappa<0>, kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[1], k_adj_kappa<1>, kBlock, 0);
    for (int k = 0; k < 2; ++k) g_adj_resident[k].store(uint32_t(std::max(per[k], 0) * std::max(sms, 0)));
}

static inline uint32_t adj_iteration_blocks(uint32_t n, int kernel) {
    uint32_t nb = adj_blocks(n), resident = g_adj_resident[kernel].load();
    return resident && resident < nb ? resident : nb;
}

void launch_adjoint_wcsph(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                          int form, const float4* pos, const float4* vel, const float* rho, const float* press,
                          const float* scaled, const float4* walls, const float4* vel_pre, const uint32_t* dest,
                          const float4* xo, const float4* vo, float4* ab, float4* xb, float4* vb, float* rb,
                          float4* xp, float4* vp, double* grads, const TerrainDev& T, const float4* slope,
                          const MoverDev& bodies, cudaStream_t s) {
    if (!p.n) return;
    uint32_t nb = adj_blocks(p.n);
    k_adj_advance<<<nb, kBlock, 0, s>>>(p, sc, vel_pre, xo, vo, ab, xb, vb, grads, pos, T);
    if (T.regions || bodies.count) {
        k_adj_force<true, true><<<adj_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, form, pos, vel, rho, press, scaled,
                                                                   walls, ab, xb, vb, rb, grads, 0, T, slope, bodies);
        k_adj_density<<<adj_blocks(p.n), kBlock, 0, s>>>(p, fl, wl, form, pos, walls, rb, xb, T.regions ? slope : nullptr,
                                                         bodies);
    } else if (p.n <= kAdjWarpMax) {
        // few rows: a warp each, so that the GPU fills
        k_adj_force_warp<<<adj_blocks(p.n * 32u), kBlock, 0, s>>>(p, sc, fl, wl, form, pos, vel, rho, press, scaled,
                                                                  walls, ab, xb, vb, rb, grads);
        k_adj_density_warp<<<adj_blocks(p.n * 32u), kBlock, 0, s>>>(p, fl, wl, form, pos, walls, rb, xb);
    } else {
        k_adj_force<true><<<adj_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, form, pos, vel, rho, press, scaled,
                                                             walls, ab, xb, vb, rb, grads, 0, T, slope, MoverDev{});
        k_adj_density<<<adj_blocks(p.n), kBlock, 0, s>>>(p, fl, wl, form, pos, walls, rb, xb, nullptr, MoverDev{});
    }
    k_adj_unsort<<<adj_blocks(p.n), kBlock, 0, s>>>(p.n, dest, xb, vb, xp, vp, nullptr, nullptr);
}



void launch_adj_advance_dfsph(const Params& p, const StepConsts* sc, const float4* vel_pre, const float4* xo,
                              const float4* vo, float4* xb, float4* w, cudaStream_t s) {
    if (p.n) k_adj_advance_dfsph<<<adj_blocks(p.n), kBlock, 0, s>>>(p, sc, vel_pre, xo, vo, xb, w);
}

void launch_adj_iteration(int which, const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                          int form, const float4* pos, const float4* walls, const float4* w, const float* rate,
                          const float* alpha, const float* rho, const float4* vel, float4* kw, float4* vr,
                          float* abar, float* rb, float4* wout, float4* xb, cudaStream_t s, int parts,
                          const float2* appbar) {
    if (!p.n) return;
    // parts: 1 the kappa pass, 2 the push, 3 both
    if ((parts & 1) && which == 1)
        k_adj_kappa<1><<<adj_iteration_blocks(p.n, 1), kBlock, 0, s>>>(p, sc, fl, wl, form, pos, walls, w, rate, alpha,
                                                          rho, vel, kw, vr, abar, rb, appbar);
    else if (parts & 1)
        k_adj_kappa<0><<<adj_iteration_blocks(p.n, 0), kBlock, 0, s>>>(p, sc, fl, wl, form, pos, walls, w, rate, alpha,
                                                          rho, vel, kw, vr, abar, rb, appbar);
    if (parts & 2)
        if (fl.gv && wl.gv)
            k_adj_push<true><<<adj_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, form, pos, walls, kw, vr, wout,
                                                                xb);
        else
            k_adj_push<false><<<adj_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, form, pos, walls, kw, vr, wout,
                                                                 xb);
}

void launch_adj_warm(int which, const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                     int form, const float4* pos, const float4* walls, const float4* w, const float2* applied,
                     const float2* appbar, float share, float4* kw, float4* vr, float2* appbar_out, float4* wout,
                     float4* xb, cudaStream_t s) {
    if (!p.n) return;
    if (which == 1)
        k_adj_warm<1><<<adj_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, form, pos, walls, w, applied, appbar, share,
                                                         kw, vr, appbar_out);
    else
        k_adj_warm<0><<<adj_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, form, pos, walls, w, applied, appbar, share,
                                                         kw, vr, appbar_out);
    launch_adj_iteration(which, p, sc, fl, wl, form, pos, walls, w, nullptr, nullptr, nullptr, nullptr, kw, vr,
                         nullptr, nullptr, wout, xb, s, 2);
}

void launch_adj_viscosity(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl, int form,
                          const float4* pos, const float4* vel, const float* rho, const float* zeros,
                          const float4* walls, float4* w, float4* ab, float4* xb, float* rb, double* grads,
                          cudaStream_t s) {
    if (!p.n) return;
    k_adj_scale<<<adj_blocks(p.n), kBlock, 0, s>>>(p, sc, w, ab, grads);
    k_adj_force<false><<<adj_blocks(p.n), kBlock, 0, s>>>(p, sc, fl, wl, form, pos, vel, rho, zeros, zeros,
                                                          walls, ab, xb, w, rb, grads, 1, TerrainDev{}, nullptr,
                                                          MoverDev{});
}

void launch_adj_factors_density(const Params& p, const PairLists& fl, const PairLists& wl, int form,
                                const float4* pos, const float4* walls, const float* alpha, const float* abar,
                                float4* gt, const float* rb, float4* xb, cudaStream_t s) {
    if (!p.n) return;
    k_adj_alpha_prep<<<adj_blocks(p.n), kBlock, 0, s>>>(p, fl, wl, form, pos, walls, alpha, abar, gt);
    k_adj_alpha<<<adj_blocks(p.n), kBlock, 0, s>>>(p, fl, wl, form, pos, walls, gt, xb);
    k_adj_density<<<adj_blocks(p.n), kBlock, 0, s>>>(p, fl, wl, form, pos, walls, rb, xb, nullptr, MoverDev{});
}

void launch_adj_unsort(uint32_t n, const uint32_t* dest, const float4* xb, const float4* vb, float4* xp, float4* vp,
                       cudaStream_t s, const float2* ib, float2* ip) {
    if (n) k_adj_unsort<<<adj_blocks(n), kBlock, 0, s>>>(n, dest, xb, vb, xp, vp, ib, ip);
}

}  // namespace slf
