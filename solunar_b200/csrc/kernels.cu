// kernels.cu -- the fluid substep on the device.
//
// One thread per particle throughout.  Particles live in SoA float4 arrays (x, y, z, unused)
// sorted by (cell, id) like the reference's arrays (src/fluid/mod.rs:540-566); every pass reads
// neighbours through the cell tables in the reference's list order, so each particle's sums are
// the reference's sequential sums, bit for bit.  Grid-wide reductions (bounding box, fastest
// particle, solver residual) are block trees feeding one atomic or one last-block finish per
// launch; the residual is summed in double-double (compensated), deterministically.
#include <atomic>
#include <cfloat>
#include <climits>

#include "fluid_device.cuh"
#include "launch.h"
#include "reduce.cuh"

namespace slf {

// Bounding box of cells, fastest speed, held-back count and non-finite flag of a block's
// particles, folded into the status with one atomic each.
__device__ __forceinline__ void fold_advance_stats(Status* st, bool valid, int3 c, float speed, uint32_t held,
                                                   uint32_t bad) {
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

// ---- bounding box and fastest speed of the current state ---------------------------------

__global__ void k_state_stats(Params p, const float4* __restrict__ pos, const float4* __restrict__ vel,
                              Status* st) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < p.n;
    int3 c = make_int3(0, 0, 0);
    float speed = 0.0f;
    if (valid) {
        float4 a = pos[i];
        float4 v = vel[i];
        c = cell_of(p, a.x, a.y, a.z);
        // Vec3::length (step.rs:92-96)
        speed = sqrtf(dot3(v.x, v.y, v.z, v.x, v.y, v.z));
        if (!(speed == speed)) speed = 0.0f;  // f32::max ignores NaN
    }
    fold_advance_stats(st, valid, c, speed, 0u, 0u);
}

// max(0, rho / rest - 1) over the particles (step.rs:84-88)
__global__ void k_max_compression(Params p, const float* __restrict__ rho, Status* st) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t b = 0;
    if (i < p.n) {
        float c = rho[i] / p.rest - 1.0f;
        if (c > 0.0f) b = __float_as_uint(c);
    }
    b = block_reduce(b, MaxU(), 0u);
    if (threadIdx.x == 0 && b) atomicMax(&st->maxcomp_bits, b);
}

// ---- spatial hash: counting sort by dense cell index, then id within each cell ------------

// cells (cell-relative positions) non-null: the cell is stored, not computed
__global__ void k_count_cells(Params p, const float4* __restrict__ pos, const int4* __restrict__ cells, int3 low,
                              int3 span, uint32_t* count, uint32_t* lin, uint32_t* slot) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    int3 c;
    if (cells) {
        int4 c4 = cells[i];
        c = make_int3(c4.x, c4.y, c4.z);
    } else {
        float4 a = pos[i];
        c = cell_of(p, a.x, a.y, a.z);
    }
    long long x = (long long)c.x - low.x, y = (long long)c.y - low.y, z = (long long)c.z - low.z;
    // the box was taken over these very positions; stay in bounds regardless
    x = x < 0 ? 0 : (x >= span.x ? span.x - 1 : x);
    y = y < 0 ? 0 : (y >= span.y ? span.y - 1 : y);
    z = z < 0 ? 0 : (z >= span.z ? span.z - 1 : z);
    uint32_t l = (uint32_t)((x * span.y + y) * span.z + z);
    lin[i] = l;
    slot[i] = atomicAdd(&count[l], 1u);
}

__global__ void k_scatter_members(uint32_t n, const uint32_t* __restrict__ lin, const uint32_t* __restrict__ slot,
                                  const uint32_t* __restrict__ start, const uint32_t* __restrict__ ids,
                                  uint32_t* members) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    members[start[lin[i]] + slot[i]] = ids[i];
}

// Final place = cell start + number of the cell's ids below this one's: the (cell, id) order
// of mod.rs:550, whatever order the atomics handed out the slots in.
__global__ void k_rank_reorder(uint32_t n, const uint32_t* __restrict__ lin, const uint32_t* __restrict__ start,
                               const uint32_t* __restrict__ members, const uint32_t* __restrict__ ids_in,
                               const float4* __restrict__ pos_in, const float4* __restrict__ vel_in,
                               const float* __restrict__ rho_in, const int4* __restrict__ cells_in,
                               uint32_t* __restrict__ ids_out, float4* __restrict__ pos_out,
                               float4* __restrict__ vel_out, float* __restrict__ rho_out,
                               int4* __restrict__ cells_out, const float2* __restrict__ warm_in,
                               float2* __restrict__ warm_out, uint32_t skip_begin, uint32_t skip_end, Status* st,
                               uint32_t* __restrict__ dest) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    // a job left undone (the fault injection of the dispatcher tests) places nothing; the count
    // of placed particles tells the host whether every particle was placed
    bool work = i < n && !(i >= skip_begin && i < skip_end);
    uint32_t placed = block_reduce(work ? 1u : 0u, SumU(), 0u);
    if (threadIdx.x == 0 && placed) atomicAdd(&st->processed, placed);
    if (!work) return;
    uint32_t l = lin[i];
    uint32_t b = start[l], e = start[l + 1];
    uint32_t id = ids_in[i];
    uint32_t rank = 0;
    for (uint32_t k = b; k < e; ++k) rank += members[k] < id ? 1u : 0u;
    uint32_t f = b + rank;
    if (dest) dest[i] = f;  // where each particle went, for the adjoint's way back
    ids_out[f] = id;
    pos_out[f] = pos_in[i];
    vel_out[f] = vel_in[i];
    rho_out[f] = rho_in[i];
    if (cells_in) cells_out[f] = cells_in[i];
    if (warm_in) warm_out[f] = warm_in[i];
}

// ---- exclusive scan of u32 in place, total written at data[m] ------------------------------

constexpr int kScanItems = 8;
constexpr int kScanTile = kBlock * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[kBlock / 32];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < kBlock / 32 ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kBlock / 32) warp_sums[lane] = s;
    }
    __syncthreads();
    uint32_t warp_prefix = warp > 0 ? warp_sums[warp - 1] : 0u;
    if (total) *total = warp_sums[kBlock / 32 - 1];
    return warp_prefix + x - v;
}

__global__ void k_scan_tiles(uint32_t* data, uint32_t m, uint32_t* tile_sums) {
    uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < m ? data[base + k] : 0u;
        sum += v[k];
    }
    uint32_t total;
    uint32_t prefix = block_exclusive_scan(sum, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < m) data[base + k] = prefix;
        prefix += v[k];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// One block scans the tile sums (any count) in place.
__global__ void k_scan_sums(uint32_t* sums, uint32_t tiles) {
    __shared__ uint32_t carry_s;
    if (threadIdx.x == 0) carry_s = 0;
    __syncthreads();
    for (uint32_t base = 0; base < tiles; base += kBlock) {
        uint32_t i = base + threadIdx.x;
        uint32_t v = i < tiles ? sums[i] : 0u;
        uint32_t total;
        uint32_t x = block_exclusive_scan(v, &total);
        uint32_t carry = carry_s;
        if (i < tiles) sums[i] = x + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry_s = carry + total;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[tiles] = carry_s;  // grand total
}

__global__ void k_scan_add(uint32_t* data, uint32_t m, const uint32_t* __restrict__ tile_sums) {
    uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t add = tile_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < m) data[base + k] += add;
    if (blockIdx.x == 0 && threadIdx.x == 0) data[m] = tile_sums[gridDim.x];
}

// ---- terrain (src/fluid/terrain.rs): the field's sampling is in fluid_device.cuh ---------------

// ground_near (mod.rs:657-663, terrain.rs:144-171, 305-310): the density the terrain regions
// holding the particle add, and the sum of their density gradients
__device__ __forceinline__ float ground_near(const TerrainDev& T, float px, float py, float pz, float3& slope) {
    float ground = 0.0f;
    slope = make_float3(0.0f, 0.0f, 0.0f);
    for (uint32_t r = 0; r < T.regions; ++r) {
        const TerrainRegion& t = T.region[r];
        float distance;
        float3 change;
        if (!terrain_read(T, t, px, py, pz, distance, change)) continue;
        float density = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
        if (distance < T.reach) {
            float open = distance - T.spacing / 2.0f;
            for (uint32_t k = 0; k < T.sites; ++k) {
                if (__ldg(&T.far[k]) <= open) continue;  // a distance moves no faster than the point
                float4 o = __ldg(&T.site[k]);
                float there;
                float3 toward;
                if (!terrain_read(T, t, px + o.x, py + o.y, pz + o.z, there, toward)) continue;
                float v = 0.5f - there / T.spacing;
                float share = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);  // solid (terrain.rs:248-250)
                density += o.w * share;
                if (share > 0.0f && share < 1.0f) {
                    float w = o.w / T.spacing;
                    gx = gx - toward.x * w;
                    gy = gy - toward.y * w;
                    gz = gz - toward.z * w;
                }
            }
        }
        ground = ground + density;
        slope = make_float3(slope.x + gx, slope.y + gy, slope.z + gz);
    }
    return ground;
}

// The second half of a list-building walk: for each of row's first m listed neighbours, in list
// order, q = pts[index] and the entry's factor becomes f(q, index, k * 32), k the entry's place
// in the list (k * 32: its offset from the row's first entry in the warp-tiled layout).  Four
// entries and their points are read ahead of their use (the entries were written by this thread
// just before: plain loads).
template <class F>
__device__ __forceinline__ void relist(const PairLists& l, uint32_t row, uint32_t m, const float4* __restrict__ pts,
                                       F&& f) {
    if (m == 0) return;
    uint2* base = l.e + l.at(row, 0);
    uint32_t j[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) j[u] = base[size_t(u < (int)m ? u : m - 1) * 32u].x;
    for (uint32_t k = 0; k < m; k += 4) {
        float4 q[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) q[u] = __ldg(&pts[j[u]]);
        uint32_t next[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            uint32_t kk = k + 4 + u;
            next[u] = base[size_t(kk < m ? kk : m - 1) * 32u].x;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k + u < m)
                base[size_t(k + u) * 32u] = make_uint2(j[u], __float_as_uint(f(q[u], j[u], (k + u) * 32u)));
#pragma unroll
        for (int u = 0; u < 4; ++u) j[u] = next[u];
    }
}

// One warp lists row `row`'s neighbours in grid g, in each_near's order: lanes 0-26 take the 27
// cells' ranges (dz outer, dy, dx inner) and sum their lengths; then 32 consecutive candidates of
// the cells laid end to end are tested at a time, a lane finding its cell by a binary search over
// the sums, and the kept ones are written in order through a ballot.  The test is each_in_cell's,
// so the list is the one-thread walk's entry for entry.  Returns the count (every lane).
__device__ __forceinline__ uint32_t warp_list_near(const Params& p, const GridDev& g, const float4* __restrict__ pts,
                                                   int3 cell, float ax, float ay, float az, const PairLists& l,
                                                   uint32_t row, uint32_t lane) {
    if (g.mode == 0) return 0u;
    uint32_t b = 0, len = 0;
    if (lane < 27u) {
        int dz = int(lane / 9u) - 1, dy = int((lane / 3u) % 3u) - 1, dx = int(lane % 3u) - 1;
        uint32_t e = 0;
        if (g.range((long long)cell.x + dx, (long long)cell.y + dy, (long long)cell.z + dz, b, e) && e > b) len = e - b;
    }
    uint32_t incl = len;  // inclusive prefix sum of the lengths over the lanes
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t up = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= uint32_t(o)) incl += up;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t m = 0;
    for (uint32_t t0 = 0; t0 < total; t0 += 32u) {
        uint32_t t = t0 + lane;
        // the first cell whose inclusive sum exceeds t (cells 0-26; lanes past the end search too)
        uint32_t lo = 0, hi = 26;
#pragma unroll
        for (int step = 0; step < 5; ++step) {
            uint32_t mid = (lo + hi) >> 1;
            uint32_t at = __shfl_sync(0xffffffffu, incl, mid);
            if (t < at) hi = mid;
            else lo = mid + 1u;
        }
        uint32_t k = lo < 26u ? lo : 26u;
        uint32_t kb = __shfl_sync(0xffffffffu, b, k), kincl = __shfl_sync(0xffffffffu, incl, k),
                 klen = __shfl_sync(0xffffffffu, len, k);
        bool keep = false;
        uint32_t j = 0;
        if (t < total) {
            j = kb + (t - (kincl - klen));
            float4 q = __ldg(&pts[j]);
            float ox = q.x - ax, oy = q.y - ay, oz = q.z - az;
            keep = dot3(ox, oy, oz, ox, oy, oz) < p.reach;
        }
        uint32_t mask = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            uint32_t at = m + __popc(mask & ((1u << lane) - 1u));
            if (at < l.cap) l.e[l.at(row, at)].x = j;
        }
        m += __popc(mask);
    }
    return m;
}

// ---- densities (mod.rs:621-675) and the substep's neighbour lists, with WCSPH pressure
// (step.rs:147-172) or the DFSPH factors (dfsph.rs:108-163) --------------------------------

// four blocks a SM (64 registers), as the pass compiled before it strode over rows
template <int SOLVER>
__global__ void __launch_bounds__(kBlock, 4) k_density(Params p, GridDev fg, GridDev wg, const float4* __restrict__ pos,
                                                    const float4* __restrict__ walls, PairLists fl, PairLists wl,
                                                    float* __restrict__ rho, float* __restrict__ press,
                                                    float* __restrict__ scaled, float* __restrict__ alpha, Status* st,
                                                    TerrainDev T, float4* __restrict__ slope, MoverDev M) {
    uint32_t compressed = 0, longest = 0;
    // rows of the walk order, a grid's width apart (one each when the grid covers them all)
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < p.n; row += gridDim.x * blockDim.x) {
        const uint32_t i = fl.particle(row);
        float4 a = pos[i];
        int3 cell = cell_of(p, a.x, a.y, a.z);
        // The walk first only lists the neighbours (a tight loop over the ~216 candidates of 27
        // cells, of which ~16 % are kept), then takes the sums over the list, in list order, so
        // the arithmetic of the kept pairs runs without the candidates' divergence.  A list over
        // its room is incomplete and the host runs the pass again with more room.
        uint32_t nf = 0, nw = 0;
        each_near(p, fg, pos, cell, a.x, a.y, a.z, [&](uint32_t j, float4) {
            if (nf < fl.cap) fl.e[fl.at(row, nf)].x = j;
            ++nf;
        });
        each_near(p, wg, walls, cell, a.x, a.y, a.z, [&](uint32_t j, float4) {
            if (nw < wl.cap) wl.e[wl.at(row, nw)].x = j;
            ++nw;
        });
        fl.count[row] = nf;
        wl.count[row] = nw;
        longest = max(longest, nf > nw ? nf : nw);
        float sum = 0.0f, wsum = 0.0f;
        float sx = 0.0f, sy = 0.0f, sz = 0.0f, squares = 0.0f;
        float4* const fgv = fl.gv ? fl.gv + fl.at(row, 0) : nullptr;
        float4* const wgv = wl.gv ? wl.gv + wl.at(row, 0) : nullptr;
        relist(fl, row, nf < fl.cap ? nf : fl.cap, pos, [&](float4 q, uint32_t j, uint32_t at) {
            float ox = q.x - a.x, oy = q.y - a.y, oz = q.z - a.z;
            float d = sqrtf(dot3(ox, oy, oz, ox, oy, oz));
            sum += kernel_value(p, d);
            float g = d <= 0.0f ? 0.0f : kernel_slope(p, d) / d;
            if (SOLVER == 1) {
                // gradient(at - other) (dfsph.rs:118), then factors (dfsph.rs:149-153)
                float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
                float gx = rx * g, gy = ry * g, gz = rz * g;
                if (fgv) fgv[at] = make_float4(gx, gy, gz, __uint_as_float(j));
                float px = gx * p.mass, py = gy * p.mass, pz = gz * p.mass;
                sx = sx + px;
                sy = sy + py;
                sz = sz + pz;
                squares += dot3(px, py, pz, px, py, pz);
            }
            return g;
        });
        relist(wl, row, nw < wl.cap ? nw : wl.cap, walls, [&](float4 q, uint32_t, uint32_t at) {
            float ox = q.x - a.x, oy = q.y - a.y, oz = q.z - a.z;
            float d = sqrtf(dot3(ox, oy, oz, ox, oy, oz));
            wsum += kernel_value(p, d);
            float g = d <= 0.0f ? 0.0f : kernel_slope(p, d) / d;
            if (SOLVER == 1) {
                float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
                float gx = rx * g, gy = ry * g, gz = rz * g;
                if (wgv) wgv[at] = make_float4(gx, gy, gz, 0.0f);
                sx = sx + gx * p.mass;
                sy = sy + gy * p.mass;
                sz = sz + gz * p.mass;
            }
            return g;
        });
        // the coupled bodies' points, in their list order (mod.rs:648-656)
        float msum = 0.0f;
        if (M.count)
            each_near(p, M.grid, M.pos, cell, a.x, a.y, a.z, [&](uint32_t, float4 q) {
                float ox = q.x - a.x, oy = q.y - a.y, oz = q.z - a.z;
                msum += kernel_value(p, sqrtf(dot3(ox, oy, oz, ox, oy, oz)));
            });
        // mass (fluid + walls + body points) + ground (mod.rs:657-663)
        float3 gslope;
        float ground = T.regions ? ground_near(T, a.x, a.y, a.z, gslope) : 0.0f;
        float density = p.mass * (sum + wsum + msum) + ground;
        rho[i] = density;
        if (slope) slope[i] = make_float4(gslope.x, gslope.y, gslope.z, 0.0f);
        if (SOLVER == 0) {
            float ratio = fminf(density / p.rest, 1.1f);
            float pressure = fmaxf(p.stiffness * (pow7(ratio) - 1.0f), 0.0f);
            press[i] = pressure;
            scaled[i] = pressure / (density * density);
        } else {
            float total = dot3(sx, sy, sz, sx, sy, sz) + squares;
            alpha[i] = total > 0.0f ? 1.0f / total : 0.0f;
        }
        float c = density / p.rest - 1.0f;
        if (c > 0.0f) compressed = max(compressed, __float_as_uint(c));
    }
    compressed = block_reduce(compressed, MaxU(), 0u);
    longest = block_reduce(longest, MaxU(), 0u);
    if (threadIdx.x == 0) {
        if (compressed) atomicMax(&st->maxcomp_bits, compressed);
        if (longest) atomicMax(&st->list_max, longest);
    }
}

// The density pass for scenes too small to fill the GPU a thread a particle: a warp a row.  The
// lists come from warp_list_near; each lane takes every 32nd listed neighbour's terms, and the
// sums run in list order, one term after the other through shuffles, so every sum and factor is
// k_density's bit for bit.  Body points and ground are taken by every lane alike.
template <int SOLVER>
__global__ void __launch_bounds__(kBlock) k_density_warp(Params p, GridDev fg, GridDev wg,
                                                         const float4* __restrict__ pos, const float4* __restrict__ walls,
                                                         PairLists fl, PairLists wl, float* __restrict__ rho,
                                                         float* __restrict__ press, float* __restrict__ scaled,
                                                         float* __restrict__ alpha, Status* st, TerrainDev T,
                                                         float4* __restrict__ slope, MoverDev M) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
    uint32_t compressed = 0, longest = 0;
    if (row < p.n) {  // whole warps
        const uint32_t i = fl.particle(row);
        const float4 a = pos[i];
        const int3 cell = cell_of(p, a.x, a.y, a.z);
        const uint32_t nf = warp_list_near(p, fg, pos, cell, a.x, a.y, a.z, fl, row, lane);
        const uint32_t nw = warp_list_near(p, wg, walls, cell, a.x, a.y, a.z, wl, row, lane);
        if (lane == 0) {
            fl.count[row] = nf;
            wl.count[row] = nw;
        }
        longest = nf > nw ? nf : nw;
        __syncwarp();  // the entries other lanes wrote
        float sum = 0.0f, wsum = 0.0f;
        float sx = 0.0f, sy = 0.0f, sz = 0.0f, squares = 0.0f;
        const uint32_t mf = nf < fl.cap ? nf : fl.cap, mw = nw < wl.cap ? nw : wl.cap;
        for (uint32_t k0 = 0; k0 < mf; k0 += 32u) {
            const uint32_t k = k0 + lane;
            float v = 0.0f, px = 0.0f, py = 0.0f, pz = 0.0f, sq = 0.0f;
            if (k < mf) {
                uint2* ent = fl.e + fl.at(row, k);
                const uint32_t j = ent->x;
                const float4 q = __ldg(&pos[j]);
                float ox = q.x - a.x, oy = q.y - a.y, oz = q.z - a.z;
                float d = sqrtf(dot3(ox, oy, oz, ox, oy, oz));
                v = kernel_value(p, d);
                float g = d <= 0.0f ? 0.0f : kernel_slope(p, d) / d;
                if (SOLVER == 1) {
                    float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
                    float gx = rx * g, gy = ry * g, gz = rz * g;
                    if (fl.gv) fl.gv[fl.at(row, k)] = make_float4(gx, gy, gz, __uint_as_float(j));
                    px = gx * p.mass, py = gy * p.mass, pz = gz * p.mass;
                    sq = dot3(px, py, pz, px, py, pz);
                }
                *ent = make_uint2(j, __float_as_uint(g));
            }
            const uint32_t here = mf - k0 < 32u ? mf - k0 : 32u;
            for (uint32_t t = 0; t < here; ++t) {
                sum += __shfl_sync(0xffffffffu, v, t);
                if (SOLVER == 1) {
                    sx = sx + __shfl_sync(0xffffffffu, px, t);
                    sy = sy + __shfl_sync(0xffffffffu, py, t);
                    sz = sz + __shfl_sync(0xffffffffu, pz, t);
                    squares += __shfl_sync(0xffffffffu, sq, t);
                }
            }
        }
        for (uint32_t k0 = 0; k0 < mw; k0 += 32u) {
            const uint32_t k = k0 + lane;
            float v = 0.0f, px = 0.0f, py = 0.0f, pz = 0.0f;
            if (k < mw) {
                uint2* ent = wl.e + wl.at(row, k);
                const uint32_t j = ent->x;
                const float4 q = __ldg(&walls[j]);
                float ox = q.x - a.x, oy = q.y - a.y, oz = q.z - a.z;
                float d = sqrtf(dot3(ox, oy, oz, ox, oy, oz));
                v = kernel_value(p, d);
                float g = d <= 0.0f ? 0.0f : kernel_slope(p, d) / d;
                if (SOLVER == 1) {
                    float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
                    float gx = rx * g, gy = ry * g, gz = rz * g;
                    if (wl.gv) wl.gv[wl.at(row, k)] = make_float4(gx, gy, gz, 0.0f);
                    px = gx * p.mass, py = gy * p.mass, pz = gz * p.mass;
                }
                *ent = make_uint2(j, __float_as_uint(g));
            }
            const uint32_t here = mw - k0 < 32u ? mw - k0 : 32u;
            for (uint32_t t = 0; t < here; ++t) {
                wsum += __shfl_sync(0xffffffffu, v, t);
                if (SOLVER == 1) {
                    sx = sx + __shfl_sync(0xffffffffu, px, t);
                    sy = sy + __shfl_sync(0xffffffffu, py, t);
                    sz = sz + __shfl_sync(0xffffffffu, pz, t);
                }
            }
        }
        // the coupled bodies' points, in their list order (mod.rs:648-656)
        float msum = 0.0f;
        if (M.count)
            each_near(p, M.grid, M.pos, cell, a.x, a.y, a.z, [&](uint32_t, float4 q) {
                float ox = q.x - a.x, oy = q.y - a.y, oz = q.z - a.z;
                msum += kernel_value(p, sqrtf(dot3(ox, oy, oz, ox, oy, oz)));
            });
        float3 gslope;
        float ground = T.regions ? ground_near(T, a.x, a.y, a.z, gslope) : 0.0f;
        float density = p.mass * (sum + wsum + msum) + ground;
        if (lane == 0) {
            rho[i] = density;
            if (slope) slope[i] = make_float4(gslope.x, gslope.y, gslope.z, 0.0f);
            if (SOLVER == 0) {
                float ratio = fminf(density / p.rest, 1.1f);
                float pressure = fmaxf(p.stiffness * (pow7(ratio) - 1.0f), 0.0f);
                press[i] = pressure;
                scaled[i] = pressure / (density * density);
            } else {
                float total = dot3(sx, sy, sz, sx, sy, sz) + squares;
                alpha[i] = total > 0.0f ? 1.0f / total : 0.0f;
            }
        }
        float c = density / p.rest - 1.0f;
        if (c > 0.0f) compressed = __float_as_uint(c);
    }
    compressed = block_reduce(compressed, MaxU(), 0u);
    longest = block_reduce(longest, MaxU(), 0u);
    if (threadIdx.x == 0) {
        if (compressed) atomicMax(&st->maxcomp_bits, compressed);
        if (longest) atomicMax(&st->list_max, longest);
    }
}

// Walks particle i's list: f(j, g, q) for each neighbour in list order, q = pts[j].  Entries are
// taken kListUnroll at a time, their gathers issued before any is used, and the next group's
// entries are requested before this group is used; past the end of the list the last entry is
// loaded again (a valid address) but not used, so the sums see exactly the list's terms in its
// order.
#ifndef SLF_LIST_UNROLL
#define SLF_LIST_UNROLL 4
#endif
constexpr int kListUnroll = SLF_LIST_UNROLL;
// resident blocks per SM the list-walking kernels are compiled for (caps their registers); the
// solver check runs best at four blocks (64 registers; 76 uncapped, three blocks)
#ifndef SLF_PAIR_MIN_BLOCKS
#define SLF_PAIR_MIN_BLOCKS 1
#endif
#ifndef SLF_RATE_MIN_BLOCKS
#define SLF_RATE_MIN_BLOCKS 4
#endif
// the push at five blocks a SM (48 registers; 56 uncapped at four blocks: 72.2 -> 70.5 us at 1M;
// six blocks spill)
#ifndef SLF_PUSH_MIN_BLOCKS
#define SLF_PUSH_MIN_BLOCKS 5
#endif



// Where a walk finds its neighbours (the global arrays, read through the L1).
struct FromGlobal {
    const float4* __restrict__ p;
    const float4* __restrict__ v;
    __device__ __forceinline__ void get(uint32_t j, float4& q) const { q = __ldg(&p[j]); }
    __device__ __forceinline__ void get(uint32_t j, float4& q, float4& w) const {
        q = __ldg(&p[j]);
        w = __ldg(&v[j]);
    }
};

template <class Src, class F>
__device__ __forceinline__ void each_listed_from(const PairLists& l, uint32_t i, const Src& src, F&& f) {
    uint32_t n = l.count[i];
    if (n > l.cap) n = l.cap;
    if (n == 0) return;
    const uint2* __restrict__ base = l.e + l.at(i, 0);
    uint2 e[kListUnroll];
#pragma unroll
    for (int u = 0; u < kListUnroll; ++u) e[u] = SLF_LIST_LOAD(base + size_t(u < (int)n ? u : n - 1) * 32u);
    for (uint32_t k = 0; k < n; k += kListUnroll) {
        float4 q[kListUnroll];
#pragma unroll
        for (int u = 0; u < kListUnroll; ++u) src.get(e[u].x, q[u]);
        uint2 next[kListUnroll];
#pragma unroll
        for (int u = 0; u < kListUnroll; ++u) {
            uint32_t kk = k + kListUnroll + u;
            next[u] = SLF_LIST_LOAD(base + size_t(kk < n ? kk : n - 1) * 32u);
        }
#pragma unroll
        for (int u = 0; u < kListUnroll; ++u)
            if (k + u < n) f(e[u].x, __uint_as_float(e[u].y), q[u]);
#pragma unroll
        for (int u = 0; u < kListUnroll; ++u) e[u] = next[u];
    }
}

template <class F>
__device__ __forceinline__ void each_listed(const PairLists& l, uint32_t i, const float4* __restrict__ pts, F&& f) {
    each_listed_from(l, i, FromGlobal{pts, nullptr}, f);
}

// The same walk with a second array gathered alongside (velocities).
template <class Src, class F>
__device__ __forceinline__ void each_listed2_from(const PairLists& l, uint32_t i, const Src& src, F&& f) {
    uint32_t n = l.count[i];
    if (n > l.cap) n = l.cap;
    if (n == 0) return;
    const uint2* __restrict__ base = l.e + l.at(i, 0);
    uint2 e[kListUnroll];
#pragma unroll
    for (int u = 0; u < kListUnroll; ++u) e[u] = SLF_LIST_LOAD(base + size_t(u < (int)n ? u : n - 1) * 32u);
    for (uint32_t k = 0; k < n; k += kListUnroll) {
        float4 q[kListUnroll], w[kListUnroll];
#pragma unroll
        for (int u = 0; u < kListUnroll; ++u) src.get(e[u].x, q[u], w[u]);
        uint2 next[kListUnroll];
#pragma unroll
        for (int u = 0; u < kListUnroll; ++u) {
            uint32_t kk = k + kListUnroll + u;
            next[u] = SLF_LIST_LOAD(base + size_t(kk < n ? kk : n - 1) * 32u);
        }
#pragma unroll
        for (int u = 0; u < kListUnroll; ++u)
            if (k + u < n) f(e[u].x, __uint_as_float(e[u].y), q[u], w[u]);
#pragma unroll
        for (int u = 0; u < kListUnroll; ++u) e[u] = next[u];
    }
}

template <class F>
__device__ __forceinline__ void each_listed2(const PairLists& l, uint32_t i, const float4* __restrict__ pts,
                                             const float4* __restrict__ more, F&& f) {
    each_listed2_from(l, i, FromGlobal{pts, more}, f);
}

// The solver check's walk over gradient entries (PairLists::gv): f(G, w) for each fluid neighbour
// in list order, G the pair's kernel gradient and w = vel[index].  Entries stream evict-first,
// kListUnroll at a time, the group's velocity gathers issued before any is used and the next
// group's entries requested before this group is used; past the end of the list the last entry
// is loaded again but not used.
template <class F>
__device__ __forceinline__ void each_gradient(const PairLists& l, uint32_t row, const float4* __restrict__ vel,
                                              F&& f) {
    uint32_t n = l.count[row];
    if (n > l.cap) n = l.cap;
    if (n == 0) return;
    const float4* __restrict__ base = l.gv + l.at(row, 0);
    float4 e[kListUnroll];
#pragma unroll
    for (int u = 0; u < kListUnroll; ++u) e[u] = SLF_LIST_LOAD(base + size_t(u < (int)n ? u : n - 1) * 32u);
    for (uint32_t k = 0; k < n; k += kListUnroll) {
        float4 w[kListUnroll];
#pragma unroll
        for (int u = 0; u < kListUnroll; ++u) w[u] = __ldg(&vel[__float_as_uint(e[u].w)]);
        float4 next[kListUnroll];
#pragma unroll
        for (int u = 0; u < kListUnroll; ++u) {
            uint32_t kk = k + kListUnroll + u;
            next[u] = SLF_LIST_LOAD(base + size_t(kk < n ? kk : n - 1) * 32u);
        }
#pragma unroll
        for (int u = 0; u < kListUnroll; ++u)
            if (k + u < n) f(e[u], w[u]);
#pragma unroll
        for (int u = 0; u < kListUnroll; ++u) e[u] = next[u];
    }
}

// The check's walk taking each slot in one of its two forms: slot k reads its kept gradient (16
// bytes, then one gather: the neighbour's velocity) when bit k % 4 of GV_SLOTS is set, and its
// {index, g} entry (8 bytes, then two gathers: position and velocity, G = (a - q) g as the
// density pass formed it) when not.  The first form moves more list bytes, the second gathers
// more: mixing them balances the pass's DRAM stream against its gathers.  f(G, w) in list order.
#ifndef SLF_RATE_GV_SLOTS
#define SLF_RATE_GV_SLOTS 0x7u
#endif
template <uint32_t GV_SLOTS, class F>
__device__ __forceinline__ void each_gradient_mixed(const PairLists& l, uint32_t row, const float4* __restrict__ pos,
                                                    const float4* __restrict__ vel, float4 a, F&& f) {
    static_assert(kListUnroll == 4, "slot forms repeat every four slots");
    uint32_t n = l.count[row];
    if (n > l.cap) n = l.cap;
    if (n == 0) return;
    const float4* __restrict__ gb = l.gv + l.at(row, 0);
    const uint2* __restrict__ eb = l.e + l.at(row, 0);
    float4 eg[4];
    uint2 ee[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        size_t kk = size_t(u < (int)n ? u : n - 1) * 32u;  // past the end: the last slot again, unused
        if (GV_SLOTS >> u & 1u) eg[u] = SLF_LIST_LOAD(gb + kk);
        else ee[u] = SLF_LIST_LOAD(eb + kk);
    }
    for (uint32_t k = 0; k < n; k += 4) {
        float4 q[4], w[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (GV_SLOTS >> u & 1u) {
                w[u] = __ldg(&vel[__float_as_uint(eg[u].w)]);
            } else {
                q[u] = __ldg(&pos[ee[u].x]);
                w[u] = __ldg(&vel[ee[u].x]);
            }
        }
        float4 ng[4];
        uint2 ne[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            uint32_t kk = k + 4 + u;
            size_t at = size_t(kk < n ? kk : n - 1) * 32u;
            if (GV_SLOTS >> u & 1u) ng[u] = SLF_LIST_LOAD(gb + at);
            else ne[u] = SLF_LIST_LOAD(eb + at);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (k + u < n) {
                if (GV_SLOTS >> u & 1u) {
                    f(eg[u], w[u]);
                } else {
                    const float g = __uint_as_float(ee[u].y);
                    const float rx = a.x - q[u].x, ry = a.y - q[u].y, rz = a.z - q[u].z;
                    f(make_float4(rx * g, ry * g, rz * g, 0.0f), w[u]);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (GV_SLOTS >> u & 1u) eg[u] = ng[u];
            else ee[u] = ne[u];
        }
    }
}

// The same over wall gradient entries, which need no gather (walls do not move): f(G).
template <class F>
__device__ __forceinline__ void each_wall_gradient(const PairLists& l, uint32_t row, F&& f) {
    uint32_t n = l.count[row];
    if (n > l.cap) n = l.cap;
    const float4* __restrict__ base = l.gv + l.at(row, 0);
#pragma unroll 4
    for (uint32_t k = 0; k < n; ++k) f(SLF_LIST_LOAD(base + size_t(k) * 32u));
}

// ---- wall viscosity (step.rs:262-301) -----------------------------------------------------

__device__ __forceinline__ float3 wall_viscous(const Params& p, float wall_visc, const PairLists& wl,
                                               const float4* __restrict__ walls, uint32_t row, float4 a, float4 v,
                                               float density, const TerrainDev& T) {
    if (wl.count[row] == 0 && T.regions == 0) return make_float3(0.0f, 0.0f, 0.0f);
    float awx = 0.0f, awy = 0.0f, awz = 0.0f;
    each_listed(wl, row, walls, [&](uint32_t, float g, float4 q) {
        float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
        awx = awx + -(rx * g);
        awy = awy + -(ry * g);
        awz = awz + -(rz * g);
    });
    // normalize_or(ZERO) dividing by the length
    float len = sqrtf(dot3(awx, awy, awz, awx, awy, awz));
    float nx = 0.0f, ny = 0.0f, nz = 0.0f;
    if (isfinite(len) && len > 0.0f) {
        nx = awx / len;
        ny = awy / len;
        nz = awz / len;
    }
    float k = fminf(dot3(v.x, v.y, v.z, nx, ny, nz), 0.0f);
    float ix = nx * k, iy = ny * k, iz = nz * k;
    float px = 0.0f, py = 0.0f, pz = 0.0f;
    // the ground damps the velocity into it by the weight of frozen water at that distance
    for (uint32_t r = 0; r < T.regions; ++r) {
        float distance;
        float3 gn;
        if (!terrain_sample(T, T.region[r], a.x, a.y, a.z, distance, gn)) continue;
        float into = dot3(v.x, v.y, v.z, gn.x, gn.y, gn.z);
        if (into < 0.0f) {
            float weight = ground_damping(T, distance);
            float c = wall_visc * into * weight / density;
            px = px - gn.x * c;
            py = py - gn.y * c;
            pz = pz - gn.z * c;
        }
    }
    each_listed(wl, row, walls, [&](uint32_t, float g, float4 q) {
        float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
        float toward = dot3(ix, iy, iz, rx, ry, rz);
        if (toward < 0.0f) {
            float squeeze = toward / (dot3(rx, ry, rz, rx, ry, rz) + p.soften);
            float damp = -wall_visc * squeeze / density;
            float s = p.mass * damp;
            px = px - (rx * g) * s;
            py = py - (ry * g) * s;
            pz = pz - (rz * g) * s;
        }
    });
    return make_float3(px, py, pz);
}

// ---- advance (step.rs:305-339) --------------------------------------------------------------

// terrain_contact (terrain.rs:314-333): each region in turn; true when the particle got under a
// surface.
__device__ __forceinline__ bool terrain_contact(const TerrainDev& T, float rest, float& nx, float& ny, float& nz,
                                                float4& v) {
    bool under = false;
    for (uint32_t r = 0; r < T.regions; ++r) contact_region(T, T.region[r], rest, nx, ny, nz, v, under);
    return under;
}

// zeroed (optional): the components the container's clamp held (bits x, y, z), whose position
// and velocity it set; terrain contact, after it, is not counted
__device__ __forceinline__ void advance_one(const Params& p, float dt, float4& a, float4& v, uint32_t& held,
                                            uint32_t& bad, const TerrainDev& T, uint32_t* zeroed = nullptr) {
    float nx = a.x + v.x * dt, ny = a.y + v.y * dt, nz = a.z + v.z * dt;
    if (p.has_bounds) {
        float ix = fminf(fmaxf(nx, p.low_in.x), p.high_in.x);
        float iy = fminf(fmaxf(ny, p.low_in.y), p.high_in.y);
        float iz = fminf(fmaxf(nz, p.low_in.z), p.high_in.z);
        if (ix != nx || iy != ny || iz != nz) {
            float cx = fminf(fmaxf(nx, p.low.x), p.high.x);
            float cy = fminf(fmaxf(ny, p.low.y), p.high.y);
            float cz = fminf(fmaxf(nz, p.low.z), p.high.z);
            if (cx != nx || cy != ny || cz != nz) held += 1;
            if (zeroed) *zeroed = (ix != nx ? 1u : 0u) | (iy != ny ? 2u : 0u) | (iz != nz ? 4u : 0u);
            if (ix != nx) v.x = 0.0f;
            if (iy != ny) v.y = 0.0f;
            if (iz != nz) v.z = 0.0f;
            nx = ix;
            ny = iy;
            nz = iz;
        }
    }
    if (T.regions && terrain_contact(T, p.spacing / 2.0f, nx, ny, nz, v)) held += 1;
    if (!(isfinite(nx) && isfinite(ny) && isfinite(nz) && isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) bad = 1;
    a.x = nx;
    a.y = ny;
    a.z = nz;
}

// ---- coupled bodies' points (couple.rs:375-416) ---------------------------------------------

// The body points within reach of a particle at `a` moving at `v`, in list order: for each,
// f(j, gradient * mass (xyz), mirrored + damp, damp, toward) with the reference's arithmetic.
template <class F>
__device__ __forceinline__ void mover_pairs(const Params& p, const MoverDev& M, float damping, float4 a, float4 v,
                                            float density, float mirrored, F&& f) {
    int3 cell = cell_of(p, a.x, a.y, a.z);
    each_near(p, M.grid, M.pos, cell, a.x, a.y, a.z, [&](uint32_t j, float4 q) {
        float ox = a.x - q.x, oy = a.y - q.y, oz = a.z - q.z;  // at - point
        float4 w = __ldg(&M.vel[j]);
        float toward = dot3(v.x - w.x, v.y - w.y, v.z - w.z, ox, oy, oz);
        float damp = toward < 0.0f ? -damping * toward / (dot3(ox, oy, oz, ox, oy, oz) + p.soften) / density : 0.0f;
        float g = kernel_gradient_factor(p, ox, oy, oz);
        f(j, (ox * g) * p.mass, (oy * g) * p.mass, (oz * g) * p.mass, mirrored + damp, damp, toward);
    });
}

// What the body points took from the water this substep: one thread per (512-particle chunk,
// body) walks the chunk's particles in order and sums, for the points of its body, the damping
// force and its torque about the body's centre (couple.rs:401-414, step.rs:173-221).  Pairs
// below the settling speed give nothing.  centre[b] = centre + moved; felt[c * bodies + b] =
// (force, torque).
// What the body points take (couple.rs:401-414) in three passes that keep the reference's order:
// each particle counts its pairs above the settling speed, a scan places them, each particle
// writes its pairs' force and torque about the owner's centre (in pair order) at its place, and
// one thread per (512-particle chunk, body) adds its body's records over the chunk's range in
// order (step.rs:173-221: chunk sums, in particle then pair order).
template <bool WRITE>
__global__ void k_mover_pairs(Params p, const StepConsts* __restrict__ sc, MoverDev M, const float4* __restrict__ pos,
                              const float4* __restrict__ vel, const float* __restrict__ rho,
                              const float* __restrict__ press, const float* __restrict__ scaled,
                              const float4* __restrict__ centre, uint32_t* __restrict__ count,
                              const uint32_t* __restrict__ offset, float4* __restrict__ pair) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    float4 a = pos[i], v = vel[i];
    float density = rho[i];
    float mirrored = scaled[i] + press[i] / p.rest_sq;
    uint32_t k = WRITE ? offset[i] : 0u;
    mover_pairs(p, M, sc->mover_damping, a, v, density, mirrored,
                [&](uint32_t j, float gx, float gy, float gz, float, float damp, float toward) {
                    float4 q = __ldg(&M.pos[j]);
                    float ox = a.x - q.x, oy = a.y - q.y, oz = a.z - q.z;
                    if (toward * toward < p.settles * dot3(ox, oy, oz, ox, oy, oz)) return;
                    if (WRITE) {
                        uint32_t b = __float_as_uint(q.w);
                        float4 o = centre[b];
                        float s = damp * p.mass;
                        float ex = gx * s, ey = gy * s, ez = gz * s;
                        float rx = q.x - o.x, ry = q.y - o.y, rz = q.z - o.z;
                        pair[2 * size_t(k)] = make_float4(ex, ey, ez, q.w);
                        pair[2 * size_t(k) + 1] =
                            make_float4(ry * ez - ey * rz, rz * ex - ez * rx, rx * ey - ex * ry, 0.0f);
                    }
                    ++k;
                });
    if (!WRITE) count[i] = k;
}

__global__ void k_mover_felt(uint32_t n, uint32_t bodies, const uint32_t* __restrict__ offset,
                             const float4* __restrict__ pair, float4* __restrict__ felt) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t chunks = (n + 511u) / 512u;
    if (t >= chunks * bodies) return;
    uint32_t c = t / bodies, b = t % bodies;
    uint32_t from = offset[c * 512u], to = offset[min(n, (c + 1u) * 512u)];
    float fx = 0.0f, fy = 0.0f, fz = 0.0f, tx = 0.0f, ty = 0.0f, tz = 0.0f;
    for (uint32_t k = from; k < to; ++k) {
        float4 f = pair[2 * size_t(k)];
        if (__float_as_uint(f.w) != b) continue;
        float4 q = pair[2 * size_t(k) + 1];
        fx = fx + f.x;
        fy = fy + f.y;
        fz = fz + f.z;
        tx = tx + q.x;
        ty = ty + q.y;
        tz = tz + q.z;
    }
    felt[2 * size_t(t)] = make_float4(fx, fy, fz, 0.0f);
    felt[2 * size_t(t) + 1] = make_float4(tx, ty, tz, 0.0f);
}

// Whether any cell of the box [lo, hi] (cell keys) holds fluid in the last sort's dense table
// (couple.rs:350-357); *wet = 1 if so.
__global__ void k_cells_wet(GridDev g, int3 lo, int3 hi, uint32_t* wet) {
    long long nx = (long long)hi.x - lo.x + 1, ny = (long long)hi.y - lo.y + 1, nz = (long long)hi.z - lo.z + 1;
    long long total = nx * ny * nz;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        long long x = lo.x + t / (ny * nz), y = lo.y + (t / nz) % ny, z = lo.z + t % nz;
        uint32_t b, e;
        if (g.range(x, y, z, b, e)) {
            *wet = 1u;
            return;
        }
    }
}

// ---- WCSPH: forces, velocity update and advance in one pass (step.rs:159-223, 305-339) -----

// Subtracts, in list order, every lane's (tx, ty, tz) of this round from (px, py, pz): lane t's
// term after lane t - 1's, as the one-thread walk subtracts them.  A lane without a term holds
// +0, whose subtraction leaves any value as it was.
__device__ __forceinline__ void take_in_order(float& px, float& py, float& pz, float tx, float ty, float tz,
                                              uint32_t here) {
    for (uint32_t t = 0; t < here; ++t) {
        px = px - __shfl_sync(0xffffffffu, tx, t);
        py = py - __shfl_sync(0xffffffffu, ty, t);
        pz = pz - __shfl_sync(0xffffffffu, tz, t);
    }
}

// The WCSPH force and advance pass for scenes too small to fill the GPU a thread a particle
// (k_density_warp made the lists): a warp a row, the pair terms a lane a neighbour, subtracted in
// list order, so every sum is k_wcsph_force's bit for bit; lane 0 advances the particle.  Without
// terrain or coupled bodies (their terms stay with k_wcsph_force).
__global__ void __launch_bounds__(kBlock) k_wcsph_force_warp(Params p, const StepConsts* __restrict__ sc, PairLists fl,
                                                             PairLists wl, const float4* __restrict__ pos,
                                                             const float4* __restrict__ vel,
                                                             const float* __restrict__ rho,
                                                             const float* __restrict__ press,
                                                             const float* __restrict__ scaled,
                                                             const float4* __restrict__ walls,
                                                             float4* __restrict__ pos_out, float4* __restrict__ vel_out,
                                                             Status* st, float4* __restrict__ vel_pre) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
    const bool valid = row < p.n;  // whole warps
    int3 nc = make_int3(0, 0, 0);
    float speed = 0.0f;
    uint32_t held = 0, bad = 0;
    if (valid) {
        const uint32_t i = fl.particle(row);
        const float dt = sc->dt;
        const float visc = sc->viscosity;
        float4 a = pos[i];
        float4 v = vel[i];
        const float density = rho[i];
        const float own = scaled[i];
        float px = 0.0f, py = 0.0f, pz = 0.0f;
        const uint32_t nf = fl.count[row], nw = wl.count[row];
        const uint32_t mf = nf < fl.cap ? nf : fl.cap, mw = nw < wl.cap ? nw : wl.cap;
        for (uint32_t k0 = 0; k0 < mf; k0 += 32u) {
            const uint32_t k = k0 + lane;
            float tx = 0.0f, ty = 0.0f, tz = 0.0f;
            if (k < mf) {
                const uint2 en = SLF_LIST_LOAD(fl.e + fl.at(row, k));
                const uint32_t j = en.x;
                const float g = __uint_as_float(en.y);
                const float4 q = __ldg(&pos[j]), w = __ldg(&vel[j]);
                float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
                float squared = dot3(rx, ry, rz, rx, ry, rz);
                if (squared > 0.0f) {
                    float gx = rx * g, gy = ry * g, gz = rz * g;
                    float toward = fminf(dot3(v.x - w.x, v.y - w.y, v.z - w.z, rx, ry, rz), 0.0f);
                    float damp = -visc * toward / (squared + p.soften) * 2.0f / (density + __ldg(&rho[j]));
                    float s = p.mass * (own + __ldg(&scaled[j]) + damp);
                    tx = gx * s, ty = gy * s, tz = gz * s;
                }
            }
            take_in_order(px, py, pz, tx, ty, tz, mf - k0 < 32u ? mf - k0 : 32u);
        }
        const float mirrored = own + press[i] / p.rest_sq;
        // the walls' pressure, then wall_viscous's two walks (its normal, then its damping)
        float awx = 0.0f, awy = 0.0f, awz = 0.0f;
        for (uint32_t k0 = 0; k0 < mw; k0 += 32u) {
            const uint32_t k = k0 + lane;
            float tx = 0.0f, ty = 0.0f, tz = 0.0f, nx = 0.0f, ny = 0.0f, nz = 0.0f;
            if (k < mw) {
                const uint2 en = SLF_LIST_LOAD(wl.e + wl.at(row, k));
                const float g = __uint_as_float(en.y);
                const float4 q = __ldg(&walls[en.x]);
                float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
                float s = p.mass * mirrored;
                tx = (rx * g) * s, ty = (ry * g) * s, tz = (rz * g) * s;
                nx = -(rx * g), ny = -(ry * g), nz = -(rz * g);
            }
            const uint32_t here = mw - k0 < 32u ? mw - k0 : 32u;
            take_in_order(px, py, pz, tx, ty, tz, here);
            for (uint32_t t = 0; t < here; ++t) {
                awx = awx + __shfl_sync(0xffffffffu, nx, t);
                awy = awy + __shfl_sync(0xffffffffu, ny, t);
                awz = awz + __shfl_sync(0xffffffffu, nz, t);
            }
        }
        float wx = 0.0f, wy = 0.0f, wz = 0.0f;
        if (nw != 0) {
            // wall_viscous (step.rs:262-301): normalize_or(ZERO) dividing by the length
            float len = sqrtf(dot3(awx, awy, awz, awx, awy, awz));
            float ux = 0.0f, uy = 0.0f, uz = 0.0f;
            if (isfinite(len) && len > 0.0f) {
                ux = awx / len;
                uy = awy / len;
                uz = awz / len;
            }
            float kk = fminf(dot3(v.x, v.y, v.z, ux, uy, uz), 0.0f);
            float ix = ux * kk, iy = uy * kk, iz = uz * kk;
            const float wall_visc = sc->wall_viscosity;
            for (uint32_t k0 = 0; k0 < mw; k0 += 32u) {
                const uint32_t k = k0 + lane;
                float tx = 0.0f, ty = 0.0f, tz = 0.0f;
                if (k < mw) {
                    const uint2 en = SLF_LIST_LOAD(wl.e + wl.at(row, k));
                    const float g = __uint_as_float(en.y);
                    const float4 q = __ldg(&walls[en.x]);
                    float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
                    float toward = dot3(ix, iy, iz, rx, ry, rz);
                    if (toward < 0.0f) {
                        float squeeze = toward / (dot3(rx, ry, rz, rx, ry, rz) + p.soften);
                        float damp = -wall_visc * squeeze / density;
                        float s = p.mass * damp;
                        tx = (rx * g) * s, ty = (ry * g) * s, tz = (rz * g) * s;
                    }
                }
                take_in_order(wx, wy, wz, tx, ty, tz, mw - k0 < 32u ? mw - k0 : 32u);
            }
        }
        if (lane == 0) {
            float ax = (px + wx) + p.gravity.x, ay = (py + wy) + p.gravity.y, az = (pz + wz) + p.gravity.z;
            v.x = v.x + ax * dt;
            v.y = v.y + ay * dt;
            v.z = v.z + az * dt;
            float4 pre = v;
            uint32_t flags = 0;
            advance_one(p, dt, a, v, held, bad, TerrainDev{}, &flags);
            if (vel_pre) {
                // the velocity before the wall zeroed any component, and which ones it zeroed
                pre.w = __uint_as_float(flags);
                vel_pre[i] = pre;
            }
            pos_out[i] = a;
            vel_out[i] = v;
            nc = cell_of(p, a.x, a.y, a.z);
            speed = sqrtf(dot3(v.x, v.y, v.z, v.x, v.y, v.z));
            if (!(speed == speed)) speed = 0.0f;
        }
    }
    fold_advance_stats(st, valid && lane == 0, nc, speed, held, bad);
}

__global__ void __launch_bounds__(kBlock, SLF_PAIR_MIN_BLOCKS) k_wcsph_force(Params p, const StepConsts* __restrict__ sc, PairLists fl,
                                                        PairLists wl, const float4* __restrict__ pos,
                                                        const float4* __restrict__ vel, const float* __restrict__ rho,
                                                        const float* __restrict__ press,
                                                        const float* __restrict__ scaled,
                                                        const float4* __restrict__ walls, float4* __restrict__ pos_out,
                                                        float4* __restrict__ vel_out, Status* st,
                                                        float4* __restrict__ vel_pre, TerrainDev T,
                                                        const float4* __restrict__ slope, MoverDev M) {
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t i = row < p.n ? fl.particle(row) : row;  // row of the walk order, its particle
    bool valid = i < p.n;
    int3 nc = make_int3(0, 0, 0);
    float speed = 0.0f;
    uint32_t held = 0, bad = 0;
    if (valid) {
        const float dt = sc->dt;
        const float visc = sc->viscosity;
        float4 a = pos[i];
        float4 v = vel[i];
        float density = rho[i];
        float own = scaled[i];
        float px = 0.0f, py = 0.0f, pz = 0.0f;
        each_listed2(fl, row, pos, vel, [&](uint32_t j, float g, float4 q, float4 w) {
            float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
            float squared = dot3(rx, ry, rz, rx, ry, rz);
            if (squared <= 0.0f) return;
            // g = slope(distance) / distance with distance = sqrt(squared) > 0
            float gx = rx * g, gy = ry * g, gz = rz * g;
            float toward = fminf(dot3(v.x - w.x, v.y - w.y, v.z - w.z, rx, ry, rz), 0.0f);
            float damp = -visc * toward / (squared + p.soften) * 2.0f / (density + __ldg(&rho[j]));
            float s = p.mass * (own + __ldg(&scaled[j]) + damp);
            px = px - gx * s;
            py = py - gy * s;
            pz = pz - gz * s;
        });
        float mirrored = own + press[i] / p.rest_sq;
        each_listed(wl, row, walls, [&](uint32_t, float g, float4 q) {
            float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
            float s = p.mass * mirrored;
            px = px - (rx * g) * s;
            py = py - (ry * g) * s;
            pz = pz - (rz * g) * s;
        });
        if (slope) {  // the ground pushes back with this particle's own pressure (step.rs:203-205)
            float4 sl = slope[i];
            px = px - sl.x * mirrored;
            py = py - sl.y * mirrored;
            pz = pz - sl.z * mirrored;
        }
        if (M.count)
            mover_pairs(p, M, sc->mover_damping, a, v, density, mirrored,
                        [&](uint32_t, float gx, float gy, float gz, float s, float, float) {
                            px = px - gx * s;
                            py = py - gy * s;
                            pz = pz - gz * s;
                        });
        float3 wv = wall_viscous(p, sc->wall_viscosity, wl, walls, row, a, v, density, T);
        float ax = (px + wv.x) + p.gravity.x, ay = (py + wv.y) + p.gravity.y, az = (pz + wv.z) + p.gravity.z;
        v.x = v.x + ax * dt;
        v.y = v.y + ay * dt;
        v.z = v.z + az * dt;
        float4 pre = v;
        uint32_t flags = 0;
        advance_one(p, dt, a, v, held, bad, T, &flags);
        if (vel_pre) {
            // the velocity before the wall zeroed any component, and which ones it zeroed
            pre.w = __uint_as_float(flags);
            vel_pre[i] = pre;
        }
        pos_out[i] = a;
        vel_out[i] = v;
        nc = cell_of(p, a.x, a.y, a.z);
        speed = sqrtf(dot3(v.x, v.y, v.z, v.x, v.y, v.z));
        if (!(speed == speed)) speed = 0.0f;
    }
    fold_advance_stats(st, valid, nc, speed, held, bad);
}

// ---- DFSPH ----------------------------------------------------------------------------------

// density_rate (dfsph.rs:166-181), then the solve's stiffness and error (dfsph.rs:241-259) of
// particle i, its neighbours taken from src.
template <int WHICH, class Src>
__device__ __forceinline__ void rate_particle(const Params& p, const StepConsts* __restrict__ sc,
                                              const PairLists& fl, const PairLists& wl, uint32_t i, uint32_t row, const Src& src,
                                              const float4* __restrict__ pos, const float4* __restrict__ vel,
                                              const float* __restrict__ rho, const float* __restrict__ alpha,
                                              const float4* __restrict__ walls, float* __restrict__ kappa_w,
                                              SolveRec rec, uint32_t slot, double& err, uint32_t& loaded) {
    const float dt = sc->dt;
    float4 a = pos[i];
    float4 v = vel[i];
    float rate = 0.0f;
    if (fl.gv && wl.gv) {
        // the gradients the density pass kept, for the slots that read them
        each_gradient_mixed<SLF_RATE_GV_SLOTS>(fl, row, pos, vel, a, [&](float4 G, float4 w) {
            rate += dot3(v.x - w.x, v.y - w.y, v.z - w.z, G.x, G.y, G.z);
        });
        each_wall_gradient(wl, row, [&](float4 G) { rate += dot3(v.x, v.y, v.z, G.x, G.y, G.z); });
    } else {
        each_listed2_from(fl, row, src, [&](uint32_t, float g, float4 q, float4 w) {
            float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
            rate += dot3(v.x - w.x, v.y - w.y, v.z - w.z, rx * g, ry * g, rz * g);
        });
        each_listed(wl, row, walls, [&](uint32_t, float g, float4 q) {
            float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
            rate += dot3(v.x, v.y, v.z, rx * g, ry * g, rz * g);
        });
    }
    rate = rate * p.mass;
    if (rec.rate) {  // recorded for the adjoint
        size_t at = size_t(slot) * p.n + i;
        rec.rate[at] = rate;
        rec.vel[at] = v;
    }
    float target, error;
    if (WHICH == 1) {
        float over = fmaxf(rho[i] + dt * rate - p.rest, 0.0f);
        target = over / sc->dt_sq;
        error = over / p.rest;
    } else {
        float r = fl.count[row] + wl.count[row] < 20u ? 0.0f : fmaxf(rate, 0.0f);
        target = r / dt;
        error = dt * r / p.rest;
    }
    // the stiffness rides in the spare lane of the position, where push_apart gathers it
    kappa_w[4 * (size_t)i + 3] = target * alpha[i];
    err = (double)error;
    loaded = error > 0.0f ? 1u : 0u;
}

// One check of the solve, a particle a thread, and the average error of the particles under
// load (dfsph.rs:263-268) in a last-block finish.
template <int WHICH>
__global__ void __launch_bounds__(kBlock, SLF_RATE_MIN_BLOCKS) k_rate(Params p, const StepConsts* __restrict__ sc, PairLists fl,
                                                 PairLists wl, const float4* __restrict__ pos,
                                                 const float4* __restrict__ vel, const float* __restrict__ rho,
                                                 const float* __restrict__ alpha, const float4* __restrict__ walls,
                                                 float* __restrict__ kappa_w, DD* __restrict__ partial,
                                                 uint32_t* __restrict__ partial_loaded, Status* st,
                                                 SolveRec rec, unsigned long long loop) {
    // a solve that already stopped leaves the rest of its batch of launches idle
    if (__ldcg(&st->settled)) return;
    DD acc{0.0, 0.0};
    uint32_t loaded = 0;
    // every block reads the count before the last block advances it
    const uint32_t slot = rec.rate ? __ldcg(&st->iterations) : 0u;
    // rows of the walk order, a grid's width apart (one each when the grid covers them all)
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < p.n; row += gridDim.x * blockDim.x) {
        const uint32_t i = fl.particle(row);
        double err = 0.0;
        uint32_t one = 0;
        rate_particle<WHICH>(p, sc, fl, wl, i, row, FromGlobal{pos, vel}, pos, vel, rho, alpha, walls, kappa_w, rec, slot,
                             err, one);
        acc = dd_add(acc, DD{err, 0.0});
        loaded += one;
    }
    residual_finish<WHICH>(p, st, partial, partial_loaded, acc, loaded, loop);
}

// push_apart (dfsph.rs:184-216) of particle i: the velocity change from each particle's
// stiffness, which the rate pass left in the w lane of each position.
template <class Src>
__device__ __forceinline__ void push_particle(const Params& p, const StepConsts* __restrict__ sc, const PairLists& fl,
                                              const PairLists& wl, uint32_t i, uint32_t row, const Src& src,
                                              const float4* __restrict__ pos, float4* __restrict__ vel,
                                              const float4* __restrict__ walls, float* __restrict__ applied) {
    const float dt = sc->dt;
    float4 a = pos[i];
    float own = a.w;
    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
    each_listed_from(fl, row, src, [&](uint32_t, float g, float4 q) {
        float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
        float s = p.mass * (own + q.w);
        cx = cx - (rx * g) * s;
        cy = cy - (ry * g) * s;
        cz = cz - (rz * g) * s;
    });
    each_listed(wl, row, walls, [&](uint32_t, float g, float4 q) {
        float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
        float s = p.mass * own;
        cx = cx - (rx * g) * s;
        cy = cy - (ry * g) * s;
        cz = cz - (rz * g) * s;
    });
    float4 v = vel[i];
    v.x = v.x + cx * dt;
    v.y = v.y + cy * dt;
    v.z = v.z + cz * dt;
    vel[i] = v;
    // warm starts: the stiffness impulse this particle's solve has applied so far
    if (applied) applied[2 * (size_t)i] += own * dt;
}

__global__ void __launch_bounds__(kBlock, SLF_PUSH_MIN_BLOCKS) k_push(Params p, const StepConsts* __restrict__ sc, PairLists fl,
                                                 PairLists wl, const float4* __restrict__ pos,
                                                 float4* __restrict__ vel, const float4* __restrict__ walls,
                                                 Status* st, float* __restrict__ applied, unsigned long long loop) {
    loop_bound(p, st, loop);
    if (__ldcg(&st->settled)) return;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < p.n; row += gridDim.x * blockDim.x)
        push_particle(p, sc, fl, wl, fl.particle(row), row, FromGlobal{pos, nullptr}, pos, vel, walls, applied);
}

// viscous (step.rs:229-251) + gravity of particle i (row `row` of the walk order)
__device__ __forceinline__ void viscous_particle(const Params& p, const StepConsts* __restrict__ sc,
                                                 const PairLists& fl, const PairLists& wl, uint32_t i, uint32_t row,
                                                 const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                 const float* __restrict__ rho, const float4* __restrict__ walls,
                                                 float4* __restrict__ vel_out) {
    const float dt = sc->dt;
    const float visc = sc->viscosity;
    float4 a = pos[i];
    float4 v = vel[i];
    float density = rho[i];
    float px = 0.0f, py = 0.0f, pz = 0.0f;
    each_listed2(fl, row, pos, vel, [&](uint32_t j, float g, float4 q, float4 w) {
        if (j == i) return;
        float rx = a.x - q.x, ry = a.y - q.y, rz = a.z - q.z;
        float toward = dot3(v.x - w.x, v.y - w.y, v.z - w.z, rx, ry, rz);
        if (toward < 0.0f) {
            float squeeze = toward / (dot3(rx, ry, rz, rx, ry, rz) + p.soften);
            float damp = -visc * squeeze * 2.0f / (density + __ldg(&rho[j]));
            float s = p.mass * damp;
            px = px - (rx * g) * s;
            py = py - (ry * g) * s;
            pz = pz - (rz * g) * s;
        }
    });
    float3 wv = wall_viscous(p, sc->wall_viscosity, wl, walls, row, a, v, density, TerrainDev{});
    float ax = (px + wv.x) + p.gravity.x, ay = (py + wv.y) + p.gravity.y, az = (pz + wv.z) + p.gravity.z;
    v.x = v.x + ax * dt;
    v.y = v.y + ay * dt;
    v.z = v.z + az * dt;
    vel_out[i] = v;
}

// viscous (step.rs:229-251) + gravity, velocity update (dfsph.rs:90-99); writes a new buffer
// because neighbours read the old velocities.
__global__ void __launch_bounds__(kBlock, SLF_PAIR_MIN_BLOCKS) k_viscous(Params p, const StepConsts* __restrict__ sc, PairLists fl,
                                                    PairLists wl, const float4* __restrict__ pos,
                                                    const float4* __restrict__ vel, const float* __restrict__ rho,
                                                    const float4* __restrict__ walls, float4* __restrict__ vel_out) {
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < p.n; row += gridDim.x * blockDim.x)
        viscous_particle(p, sc, fl, wl, fl.particle(row), row, pos, vel, rho, walls, vel_out);
}

__global__ void k_advance(Params p, const StepConsts* __restrict__ sc, const float4* __restrict__ pos_in,
                          float4* __restrict__ pos_out, float4* __restrict__ vel, Status* st,
                          float4* __restrict__ vel_pre) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < p.n;
    int3 nc = make_int3(0, 0, 0);
    float speed = 0.0f;
    uint32_t held = 0, bad = 0;
    if (valid) {
        float4 a = pos_in[i];
        float4 v = vel[i];
        float4 pre = v;
        uint32_t flags = 0;
        advance_one(p, sc->dt, a, v, held, bad, TerrainDev{}, &flags);
        if (vel_pre) {
            pre.w = __uint_as_float(flags);
            vel_pre[i] = pre;
        }
        pos_out[i] = a;
        vel[i] = v;
        nc = cell_of(p, a.x, a.y, a.z);
        speed = sqrtf(dot3(v.x, v.y, v.z, v.x, v.y, v.z));
        if (!(speed == speed)) speed = 0.0f;
    }
    fold_advance_stats(st, valid, nc, speed, held, bad);
}

// ---- neighbour lists on demand (mod.rs:570-606) --------------------------------------------

__global__ void k_list_count(Params p, GridDev g, const float4* __restrict__ pos, const float4* __restrict__ pts,
                             uint32_t* counts) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    float4 a = pos[i];
    int3 cell = cell_of(p, a.x, a.y, a.z);
    uint32_t c = 0;
    each_near(p, g, pts, cell, a.x, a.y, a.z, [&](uint32_t, float4) { ++c; });
    counts[i] = c;
}

__global__ void k_list_fill(Params p, GridDev g, const float4* __restrict__ pos, const float4* __restrict__ pts,
                            const uint32_t* __restrict__ start, uint32_t* items) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    float4 a = pos[i];
    int3 cell = cell_of(p, a.x, a.y, a.z);
    uint32_t k = start[i];
    each_near(p, g, pts, cell, a.x, a.y, a.z, [&](uint32_t j, float4) { items[k++] = j; });
}

// ---- the walk order of the list passes (PairLists::order) -------------------------------------
// Cells taken in 2 x 2-column bricks, so 256 consecutive rows cover about 2 x 2 x 8 cells instead
// of a 1 x 1 x 32 column.  SLF_WALK_ZQUAD 0: key = ((x / 2, y / 2), z, x % 2, y % 2); 1: the
// brick's z split in quads, key = ((x / 2, y / 2), z / 4, x % 2, y % 2, z % 4), so a warp's 32
// rows are (about) four consecutive cells of one column, whose neighbours lie in consecutive
// cells of the same neighbouring columns: a warp's gathers touch fewer cache lines.
#ifndef SLF_WALK_ZQUAD
#define SLF_WALK_ZQUAD 1
#endif

__host__ __device__ __forceinline__ uint32_t walk_quads(int z) { return SLF_WALK_ZQUAD ? (uint32_t(z) + 3u) / 4u : uint32_t(z); }

__device__ __forceinline__ uint32_t brick_key(uint32_t lin, int3 span) {
    uint32_t z = lin % (uint32_t)span.z, xy = lin / (uint32_t)span.z;
    uint32_t y = xy % (uint32_t)span.y, x = xy / (uint32_t)span.y;
    uint32_t by = ((uint32_t)span.y + 1u) / 2u;
    if (SLF_WALK_ZQUAD)
        return ((((x >> 1) * by + (y >> 1)) * walk_quads(span.z) + (z >> 2)) * 4u + (x & 1u) * 2u + (y & 1u)) * 4u +
               (z & 3u);
    return (((x >> 1) * by + (y >> 1)) * (uint32_t)span.z + z) * 4u + (x & 1u) * 2u + (y & 1u);
}

// bcount[key(cell)] = members of the cell (bcount cleared beforehand: keys of the padding stay 0)
__global__ void k_brick_count(uint32_t volume, int3 span, const uint32_t* __restrict__ start,
                              uint32_t* __restrict__ bcount) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= volume) return;
    bcount[brick_key(c, span)] = start[c + 1] - start[c];
}

// each cell's members, contiguous in the sorted arrays, go to the rows its key's scan names
__global__ void k_brick_fill(uint32_t volume, int3 span, const uint32_t* __restrict__ start,
                             const uint32_t* __restrict__ bstart, uint32_t* __restrict__ order) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= volume) return;
    uint32_t b = start[c], e = start[c + 1], r = bstart[brick_key(c, span)];
    for (uint32_t m = b; m < e; ++m) order[r + (m - b)] = m;
}

// ---- domain (mod.rs:451-486): keep flags, then a stable compaction -------------------------

// The f32 position the readouts give: cell-relative ones rebuilt in double and rounded once.
__device__ __forceinline__ float4 absolute_of(const Params& p, const float4* __restrict__ pos,
                                              const int4* __restrict__ cells, uint32_t i) {
    float4 a = pos[i];
    if (cells) {
        int4 c = cells[i];
        const double r = p.radius;
        a.x = float(double(c.x) * r + a.x);
        a.y = float(double(c.y) * r + a.y);
        a.z = float(double(c.z) * r + a.z);
    }
    return a;
}

// drain = 0: keep what the domain holds, clamp(p) == p (mod.rs:451-486); drain = 1: keep what
// lies outside the drain box, inclusive bounds (flow.rs:154-161)
__global__ void k_domain_flags(Params p, const float4* __restrict__ pos, const int4* __restrict__ cells, float3 low,
                               float3 high, int drain, uint32_t* keep) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    float4 a = absolute_of(p, pos, cells, i);
    if (drain) {
        bool inside = a.x >= low.x && a.y >= low.y && a.z >= low.z && a.x <= high.x && a.y <= high.y && a.z <= high.z;
        keep[i] = inside ? 0u : 1u;
        return;
    }
    float cx = fminf(fmaxf(a.x, low.x), high.x), cy = fminf(fmaxf(a.y, low.y), high.y),
          cz = fminf(fmaxf(a.z, low.z), high.z);
    keep[i] = (cx == a.x && cy == a.y && cz == a.z) ? 1u : 0u;
}

// ---- emitters (flow.rs:168-226) --------------------------------------------------------------
// Lattice slots of an emitter box: cnt per axis, slot (x, y, z) at index (y cnt.z + z) cnt.x + x,
// its centre low + ((x, y, z) + 1/2) spacing.  A slot is taken when a particle is nearer its
// centre than 0.9 spacing; each particle tests the 3 x 3 x 3 slots around its nearest one.

// Rust's `f as i64` (saturating, NaN to 0), then held to [-2, cells + 1]: further out reaches no slot
__device__ __forceinline__ long long nearest_slot(float v, int cells) {
    float r = roundf(v);
    long long c = (r != r) ? 0 : (r >= 9.2233720e18f ? LLONG_MAX : (r <= -9.2233720e18f ? LLONG_MIN : (long long)r));
    return c < -2 ? -2 : (c > cells + 1 ? cells + 1 : c);
}

__global__ void k_emitter_taken(Params p, const float4* __restrict__ pos, const int4* __restrict__ cells, float3 low,
                                int3 cnt, float spacing, float clear, uint32_t* __restrict__ taken) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    float4 a = absolute_of(p, pos, cells, i);
    long long nx = nearest_slot((a.x - low.x) / spacing - 0.5f, cnt.x);
    long long ny = nearest_slot((a.y - low.y) / spacing - 0.5f, cnt.y);
    long long nz = nearest_slot((a.z - low.z) / spacing - 0.5f, cnt.z);
    for (long long y = ny - 1; y <= ny + 1; ++y)
        for (long long z = nz - 1; z <= nz + 1; ++z)
            for (long long x = nx - 1; x <= nx + 1; ++x) {
                if (x < 0 || x >= cnt.x || y < 0 || y >= cnt.y || z < 0 || z >= cnt.z) continue;
                float ox = a.x - (low.x + (float(x) + 0.5f) * spacing);
                float oy = a.y - (low.y + (float(y) + 0.5f) * spacing);
                float oz = a.z - (low.z + (float(z) + 0.5f) * spacing);
                if (dot3(ox, oy, oz, ox, oy, oz) < clear) taken[(y * cnt.z + z) * cnt.x + x] = 1u;
            }
}

// After an exclusive scan of `taken` (total at taken_ex[total]): the free slots in slot order
// become particles first_id, first_id + 1, ... until `room` of them are placed.
__global__ void k_emit(uint32_t total, const uint32_t* __restrict__ taken_ex, int3 cnt, float3 low, float spacing,
                       float3 velocity, uint32_t room, uint32_t first_id, float4* __restrict__ pos_out,
                       float4* __restrict__ vel_out, uint32_t* __restrict__ ids_out, float* __restrict__ rho_out) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= total || taken_ex[s + 1] != taken_ex[s]) return;
    uint32_t rank = s - taken_ex[s];
    if (rank >= room) return;
    uint32_t x = s % uint32_t(cnt.x), z = (s / uint32_t(cnt.x)) % uint32_t(cnt.z), y = s / (uint32_t(cnt.x) * uint32_t(cnt.z));
    pos_out[rank] = make_float4(low.x + (float(x) + 0.5f) * spacing, low.y + (float(y) + 0.5f) * spacing,
                                low.z + (float(z) + 0.5f) * spacing, 0.0f);
    vel_out[rank] = make_float4(velocity.x, velocity.y, velocity.z, 0.0f);
    ids_out[rank] = first_id + rank;
    rho_out[rank] = 0.0f;
}

__global__ void k_compact(uint32_t n, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ dest,
                          const uint32_t* __restrict__ ids_in, const float4* __restrict__ pos_in,
                          const float4* __restrict__ vel_in, const float* __restrict__ rho_in,
                          const int4* __restrict__ cells_in, uint32_t* __restrict__ ids_out,
                          float4* __restrict__ pos_out, float4* __restrict__ vel_out, float* __restrict__ rho_out,
                          int4* __restrict__ cells_out, const float2* __restrict__ warm_in,
                          float2* __restrict__ warm_out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !keep[i]) return;
    uint32_t f = dest[i];
    ids_out[f] = ids_in[i];
    pos_out[f] = pos_in[i];
    vel_out[f] = vel_in[i];
    rho_out[f] = rho_in[i];
    if (cells_in) cells_out[f] = cells_in[i];
    if (warm_in) warm_out[f] = warm_in[i];
}

// ---- carrying the body points through a step (couple.rs:291-318) -----------------------------

// The points at `elapsed` (start + velocity * elapsed, owner bits in start.w) and their place in
// the dense table of box (low, span): lin[i], and slot[i] among the cell's points counted so far.
__global__ void k_mover_cells(Params p, uint32_t k, const float4* __restrict__ start, const float4* __restrict__ vel,
                              float elapsed, int3 low, int3 span, uint32_t* __restrict__ lin,
                              uint32_t* __restrict__ slot, uint32_t* __restrict__ count) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    const float4 s0 = start[i], v = vel[i];
    const float x = s0.x + v.x * elapsed, y = s0.y + v.y * elapsed, z = s0.z + v.z * elapsed;
    const int3 c = cell_of(p, x, y, z);
    const uint32_t l = uint32_t(((long long)(c.x - low.x) * span.y + (c.y - low.y)) * span.z + (c.z - low.z));
    lin[i] = l;
    slot[i] = atomicAdd(&count[l], 1u);
}

// The points sorted by (cell, owner, place in the current order), as the host sort of
// couple.rs:291-318 orders them: a point's place in its cell is the number of the cell's points
// with a smaller (owner, current place).  Writes the sorted starts, velocities and positions at
// `elapsed` (owner bits in w).
__global__ void k_mover_order(uint32_t k, const uint32_t* __restrict__ lin, const uint32_t* __restrict__ slot,
                              const uint32_t* __restrict__ table, uint32_t* __restrict__ members,
                              const float4* __restrict__ start, const float4* __restrict__ vel, float elapsed,
                              float4* __restrict__ start_out, float4* __restrict__ vel_out,
                              float4* __restrict__ pos_out, int phase) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    const uint32_t l = lin[i], b = table[l];
    if (phase == 0) {  // the cell's members, in any order
        members[b + slot[i]] = i;
        return;
    }
    const uint32_t e = table[l + 1];
    const uint32_t own = __float_as_uint(start[i].w);
    uint32_t rank = 0;
    for (uint32_t q = b; q < e; ++q) {
        const uint32_t m = members[q];
        const uint32_t om = __float_as_uint(__ldg(&start[m].w));
        rank += (om < own || (om == own && m < i)) ? 1u : 0u;
    }
    const uint32_t d = b + rank;
    const float4 s0 = start[i], v = vel[i];
    start_out[d] = s0;
    vel_out[d] = v;
    pos_out[d] = make_float4(s0.x + v.x * elapsed, s0.y + v.y * elapsed, s0.z + v.z * elapsed, s0.w);
}

// ---- the particles a coupled body's lift reads (lift.rs:29-60) -----------------------------------

// keep[i] = 1 for a particle inside any of the boxes (low, high pairs, bounds inclusive, NaN
// bounds ignored and NaN positions outside, as the host's clamp test min(max(p, low), high) == p)
__global__ void k_in_boxes(uint32_t n, const float4* __restrict__ pos, const float3* __restrict__ boxes,
                           uint32_t count, uint32_t* __restrict__ keep) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = pos[i];
    uint32_t in = 0;
    if (a.x == a.x && a.y == a.y && a.z == a.z) {
        for (uint32_t b = 0; b < count && !in; ++b) {
            const float3 lo = boxes[2 * b], hi = boxes[2 * b + 1];
            in = !(lo.x > a.x) && !(a.x > hi.x) && !(lo.y > a.y) && !(a.y > hi.y) && !(lo.z > a.z) && !(a.z > hi.z);
        }
    }
    keep[i] = in;
}

// the kept particles in index order: their index, position and velocity (xyz, 6 floats)
__global__ void k_gather_kept(uint32_t n, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ at,
                              const float4* __restrict__ pos, const float4* __restrict__ vel,
                              uint32_t* __restrict__ index, float* __restrict__ pv) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !keep[i]) return;
    const uint32_t k = at[i];
    const float4 a = pos[i], v = vel[i];
    index[k] = i;
    float* o = pv + 6 * size_t(k);
    o[0] = a.x;
    o[1] = a.y;
    o[2] = a.z;
    o[3] = v.x;
    o[4] = v.y;
    o[5] = v.z;
}

// vel[index[k]].xyz = v3[k]
__global__ void k_scatter_velocities(uint32_t m, const uint32_t* __restrict__ index, const float* __restrict__ v3,
                                     float4* __restrict__ vel) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const uint32_t i = index[k];
    vel[i] = make_float4(v3[3 * size_t(k)], v3[3 * size_t(k) + 1], v3[3 * size_t(k) + 2], 0.0f);
}

__global__ void k_set_consts(StepConsts c, StepConsts* out) { *out = c; }

// xyz triples <-> float4, so host copies move 12 bytes a particle
__global__ void k_pack3(uint32_t n, const float4* __restrict__ in, float* __restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = in[i];
    out[3 * i] = v.x;
    out[3 * i + 1] = v.y;
    out[3 * i + 2] = v.z;
}

// xyz triples into float4 slots; `bad` (optional) counts triples with a non finite component
__global__ void k_unpack3(uint32_t n, const float* __restrict__ in, float4* __restrict__ out, uint32_t* bad) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = in[3 * i], y = in[3 * i + 1], z = in[3 * i + 2];
    if (bad && !(isfinite(x) && isfinite(y) && isfinite(z))) atomicAdd(bad, 1u);
    out[i] = make_float4(x, y, z, 0.0f);
}

// ---- launchers ------------------------------------------------------------------------------

static std::atomic<uint64_t> g_launches{0};
uint64_t kernel_launches() { return g_launches.load(); }
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void note_launches(int64_t k) { g_launches.fetch_add(uint64_t(k), std::memory_order_relaxed); }

static inline uint32_t blocks_for(uint32_t n) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return (n + kBlock - 1) / kBlock;
}

// The list passes' grids (the solves' check and push, the density pass, the viscosity): with
// SLF_SOLVER_RESIDENT, no more blocks than the SMs hold at once (each block then strides over
// rows), so no launch ends on a partial wave and the check's residual sums fewer block partials.
#ifndef SLF_SOLVER_RESIDENT
#define SLF_SOLVER_RESIDENT 1
#endif
// resident blocks of k_rate<0>, k_rate<1>, k_push, k_density<0>, k_density<1>, k_viscous on the
// device (prepare_solver_grids; 0: not known yet, the grid then covers every row)
static std::atomic<uint32_t> g_resident[6] = {0, 0, 0, 0, 0, 0};

void prepare_solver_grids() {
    if (!SLF_SOLVER_RESIDENT || g_resident[2].load()) return;
    int dev = 0, sms = 0, per[6] = {0, 0, 0, 0, 0, 0};
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[0], k_rate<0>, kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[1], k_rate<1>, kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[2], k_push, kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[3], k_density<0>, kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[4], k_density<1>, kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per[5], k_viscous, kBlock, 0);
    for (int k = 0; k < 6; ++k) g_resident[k].store(uint32_t(std::max(per[k], 0) * std::max(sms, 0)));
}

static uint32_t solver_blocks(uint32_t n, int kernel) {
    uint32_t nb = blocks_for(n);
    uint32_t resident = g_resident[kernel].load();
    return resident && resident < nb ? resident : nb;
}

void launch_pack3(uint32_t n, const float4* in, float* out, cudaStream_t s) {
    if (n) k_pack3<<<blocks_for(n), kBlock, 0, s>>>(n, in, out);
}

void launch_unpack3(uint32_t n, const float* in, float4* out, cudaStream_t s, uint32_t* bad) {
    if (n) k_unpack3<<<blocks_for(n), kBlock, 0, s>>>(n, in, out, bad);
}

void launch_state_stats(const Params& p, const float4* pos, const float4* vel, Status* st, cudaStream_t s) {
    if (p.n) k_state_stats<<<blocks_for(p.n), kBlock, 0, s>>>(p, pos, vel, st);
}

void launch_max_compression(const Params& p, const float* rho, Status* st, cudaStream_t s) {
    if (p.n) k_max_compression<<<blocks_for(p.n), kBlock, 0, s>>>(p, rho, st);
}

void launch_count_cells(const Params& p, const float4* pos, const int4* cells, int3 low, int3 span, uint32_t* count,
                        uint32_t* lin, uint32_t* slot, cudaStream_t s) {
    if (p.n) k_count_cells<<<blocks_for(p.n), kBlock, 0, s>>>(p, pos, cells, low, span, count, lin, slot);
}

size_t scan_tiles(uint32_t m) { return (m + kScanTile - 1) / kScanTile; }

void launch_exclusive_scan(uint32_t* data, uint32_t m, uint32_t* tile_sums, cudaStream_t s) {
    if (m == 0) return;
    uint32_t tiles = (uint32_t)scan_tiles(m);
    g_launches.fetch_add(3, std::memory_order_relaxed);
    k_scan_tiles<<<tiles, kBlock, 0, s>>>(data, m, tile_sums);
    k_scan_sums<<<1, kBlock, 0, s>>>(tile_sums, tiles);
    k_scan_add<<<tiles, kBlock, 0, s>>>(data, m, tile_sums);
}

void launch_scatter_members(uint32_t n, const uint32_t* lin, const uint32_t* slot, const uint32_t* start,
                            const uint32_t* ids, uint32_t* members, cudaStream_t s) {
    if (n) k_scatter_members<<<blocks_for(n), kBlock, 0, s>>>(n, lin, slot, start, ids, members);
}

void launch_rank_reorder(uint32_t n, const uint32_t* lin, const uint32_t* start, const uint32_t* members,
                         const uint32_t* ids_in, const float4* pos_in, const float4* vel_in, const float* rho_in,
                         const int4* cells_in, uint32_t* ids_out, float4* pos_out, float4* vel_out, float* rho_out,
                         int4* cells_out, const float2* warm_in, float2* warm_out, uint32_t skip_begin,
                         uint32_t skip_end, Status* st, uint32_t* dest,
                         cudaStream_t s) {
    if (n)
        k_rank_reorder<<<blocks_for(n), kBlock, 0, s>>>(n, lin, start, members, ids_in, pos_in, vel_in, rho_in,
                                                        cells_in, ids_out, pos_out, vel_out, rho_out, cells_out,
                                                        warm_in, warm_out,
                                                        skip_begin, skip_end, st, dest);
}

void launch_density(const Params& p, const GridDev& fg, const GridDev& wg, const float4* pos, const float4* walls,
                    const PairLists& fl, const PairLists& wl, float* rho, float* press, float* scaled, float* alpha,
                    Status* st, const TerrainDev& T, float4* slope, cudaStream_t s, const MoverDev& M) {
    if (!p.n) return;
    if (warp_rows(p.n, p.radius, p.spacing) && T.regions == 0 && M.count == 0) {
        // a scene this small leaves most SMs idle a thread a particle: a warp a particle (terrain
        // and body points, which every lane would take alike, stay a thread a particle)
        if (p.solver == 0)
            k_density_warp<0><<<blocks_for(p.n * 32u), kBlock, 0, s>>>(p, fg, wg, pos, walls, fl, wl, rho, press,
                                                                       scaled, alpha, st, T, slope, M);
        else
            k_density_warp<1><<<blocks_for(p.n * 32u), kBlock, 0, s>>>(p, fg, wg, pos, walls, fl, wl, rho, press,
                                                                       scaled, alpha, st, T, slope, M);
        return;
    }
    if (p.solver == 0)
        k_density<0><<<solver_blocks(p.n, 3), kBlock, 0, s>>>(p, fg, wg, pos, walls, fl, wl, rho, press, scaled, alpha, st,
                                                        T, slope, M);
    else
        k_density<1><<<solver_blocks(p.n, 4), kBlock, 0, s>>>(p, fg, wg, pos, walls, fl, wl, rho, press, scaled, alpha, st,
                                                        T, slope, M);
}

void launch_wcsph_force(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                        const float4* pos, const float4* vel, const float* rho, const float* press,
                        const float* scaled, const float4* walls, float4* pos_out, float4* vel_out, Status* st,
                        float4* vel_pre, const TerrainDev& T, const float4* slope, cudaStream_t s,
                        const MoverDev& M) {
    if (!p.n) return;
    if (warp_rows(p.n, p.radius, p.spacing) && T.regions == 0 && M.count == 0 && slope == nullptr) {
        k_wcsph_force_warp<<<blocks_for(p.n * 32u), kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, press, scaled,
                                                                    walls, pos_out, vel_out, st, vel_pre);
        return;
    }
    k_wcsph_force<<<blocks_for(p.n), kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, press, scaled, walls, pos_out,
                                                     vel_out, st, vel_pre, T, slope, M);
}

void launch_mover_count(const Params& p, const StepConsts* sc, const MoverDev& M, const float4* pos,
                        const float4* vel, const float* rho, const float* press, const float* scaled,
                        uint32_t* count, cudaStream_t s) {
    if (p.n)
        k_mover_pairs<false><<<blocks_for(p.n), kBlock, 0, s>>>(p, sc, M, pos, vel, rho, press, scaled, nullptr, count,
                                                                nullptr, nullptr);
}

void launch_mover_felt(const Params& p, const StepConsts* sc, const MoverDev& M, const float4* pos, const float4* vel,
                       const float* rho, const float* press, const float* scaled, const float4* centre,
                       uint32_t bodies, const uint32_t* offset, float4* pair, float4* felt, cudaStream_t s) {
    if (!p.n) return;
    k_mover_pairs<true><<<blocks_for(p.n), kBlock, 0, s>>>(p, sc, M, pos, vel, rho, press, scaled, centre, nullptr,
                                                           offset, pair);
    uint32_t threads = (p.n + 511u) / 512u * bodies;
    if (threads) k_mover_felt<<<(threads + 63u) / 64u, 64, 0, s>>>(p.n, bodies, offset, pair, felt);
    note_launch();
}

// What each body took this substep, folded into its step's impulse as the host folds it
// (step.rs:173-221): chunk by chunk in order, impulse + force * dt, angular + torque * dt.  A block
// a body: its threads bring the chunks' records into shared memory 256 at a time and one thread
// adds them in order.
__global__ void k_mover_fold(uint32_t chunks, uint32_t bodies, const float4* __restrict__ felt, float dt,
                             float4* __restrict__ impulse) {
    __shared__ float4 force[kBlock], torque[kBlock];
    const uint32_t b = blockIdx.x, t = threadIdx.x;
    float4 imp = impulse[2 * size_t(b)], ang = impulse[2 * size_t(b) + 1];
    for (uint32_t base = 0; base < chunks; base += kBlock) {
        const uint32_t c = base + t;
        if (c < chunks) {
            force[t] = felt[2 * (size_t(c) * bodies + b)];
            torque[t] = felt[2 * (size_t(c) * bodies + b) + 1];
        }
        __syncthreads();
        if (t == 0) {
            const uint32_t here = chunks - base < uint32_t(kBlock) ? chunks - base : uint32_t(kBlock);
#pragma unroll 8
            for (uint32_t j = 0; j < here; ++j) {
                const float4 f = force[j], q = torque[j];
                imp = make_float4(imp.x + f.x * dt, imp.y + f.y * dt, imp.z + f.z * dt, 0.0f);
                ang = make_float4(ang.x + q.x * dt, ang.y + q.y * dt, ang.z + q.z * dt, 0.0f);
            }
        }
        __syncthreads();
    }
    if (t == 0) {
        impulse[2 * size_t(b)] = imp;
        impulse[2 * size_t(b) + 1] = ang;
    }
}

void launch_mover_fold(uint32_t n, uint32_t bodies, const float4* felt, float dt, float4* impulse, cudaStream_t s) {
    if (!n || !bodies) return;
    k_mover_fold<<<bodies, kBlock, 0, s>>>((n + 511u) / 512u, bodies, felt, dt, impulse);
    note_launch();
}

void launch_cells_wet(const GridDev& g, int3 lo, int3 hi, uint32_t* wet, cudaStream_t s) {
    long long total = ((long long)hi.x - lo.x + 1) * ((long long)hi.y - lo.y + 1) * ((long long)hi.z - lo.z + 1);
    if (total <= 0) return;
    long long blocks = std::min<long long>((total + kBlock - 1) / kBlock, 4096);
    k_cells_wet<<<uint32_t(blocks), kBlock, 0, s>>>(g, lo, hi, wet);
    note_launch();
}

size_t rate_partial_bytes(uint32_t n) { return (n + kBlock - 1) / kBlock * (sizeof(DD) + sizeof(uint32_t)) + 64; }


void launch_rate(int which, const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl,
                 float4* pos, const float4* vel, const float* rho, const float* alpha, const float4* walls,
                 void* partials, Status* st, SolveRec rec, cudaStream_t s, unsigned long long loop) {
    if (!p.n) return;
    // the partials' room is for one block a 256 rows; the grid takes at most that many
    uint32_t nb = solver_blocks(p.n, which == 0 ? 0 : 1);
    DD* part = static_cast<DD*>(partials);
    uint32_t* loaded = reinterpret_cast<uint32_t*>(part + (p.n + kBlock - 1) / kBlock);
    if (which == 0)
        k_rate<0><<<nb, kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, alpha, walls, reinterpret_cast<float*>(pos),
                                        part, loaded, st, rec, loop);
    else
        k_rate<1><<<nb, kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, alpha, walls, reinterpret_cast<float*>(pos),
                                        part, loaded, st, rec, loop);
}

void launch_push(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl, const float4* pos,
                 float4* vel, const float4* walls, Status* st, float* applied, cudaStream_t s, unsigned long long loop) {
    if (p.n) k_push<<<solver_blocks(p.n, 2), kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, walls, st, applied, loop);
}

// Warm start of a solve: the stiffness that applies `share` of the impulse S the particle's last
// solve of this kind applied (S = sum of kappa dt), at this substep's dt, into the position's
// spare lane for one push; S restarts from that push's impulse.
__global__ void k_warm_kappa(Params p, const StepConsts* __restrict__ sc, float share, float* __restrict__ applied,
                             float4* __restrict__ pos) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const float dt = sc->dt;
    float kappa = share * applied[2 * (size_t)i] / dt;
    pos[i].w = kappa;
    applied[2 * (size_t)i] = kappa * dt;
}

void launch_warm_kappa(const Params& p, const StepConsts* sc, float share, float* applied, float4* pos, cudaStream_t s) {
    if (p.n) k_warm_kappa<<<blocks_for(p.n), kBlock, 0, s>>>(p, sc, share, applied, pos);
}

size_t walk_order_keys(int3 span) {
    return size_t((span.x + 1) / 2) * size_t((span.y + 1) / 2) * size_t(walk_quads(span.z)) * (SLF_WALK_ZQUAD ? 16u : 4u);
}

void launch_walk_order(uint32_t volume, int3 span, const uint32_t* start, uint32_t* bcount, uint32_t* tile_sums,
                       uint32_t* order, cudaStream_t s) {
    if (!volume) return;
    size_t keys = walk_order_keys(span);
    cudaMemsetAsync(bcount, 0, (keys + 1) * sizeof(uint32_t), s);
    k_brick_count<<<blocks_for(volume), kBlock, 0, s>>>(volume, span, start, bcount);
    launch_exclusive_scan(bcount, uint32_t(keys), tile_sums, s);
    k_brick_fill<<<blocks_for(volume), kBlock, 0, s>>>(volume, span, start, bcount, order);
}

void launch_viscous(const Params& p, const StepConsts* sc, const PairLists& fl, const PairLists& wl, const float4* pos,
                    const float4* vel, const float* rho, const float4* walls, float4* vel_out, cudaStream_t s) {
    if (p.n) k_viscous<<<solver_blocks(p.n, 5), kBlock, 0, s>>>(p, sc, fl, wl, pos, vel, rho, walls, vel_out);
}

void launch_advance(const Params& p, const StepConsts* sc, const float4* pos_in, float4* pos_out, float4* vel,
                    Status* st, float4* vel_pre, cudaStream_t s) {
    if (p.n) k_advance<<<blocks_for(p.n), kBlock, 0, s>>>(p, sc, pos_in, pos_out, vel, st, vel_pre);
}

void launch_list_count(const Params& p, const GridDev& g, const float4* pos, const float4* pts, uint32_t* counts,
                       cudaStream_t s) {
    if (p.n) k_list_count<<<blocks_for(p.n), kBlock, 0, s>>>(p, g, pos, pts, counts);
}

void launch_list_fill(const Params& p, const GridDev& g, const float4* pos, const float4* pts, const uint32_t* start,
                      uint32_t* items, cudaStream_t s) {
    if (p.n) k_list_fill<<<blocks_for(p.n), kBlock, 0, s>>>(p, g, pos, pts, start, items);
}

void launch_emitter_taken(const Params& p, const float4* pos, const int4* cells, float3 low, int3 cnt, float spacing,
                          float clear, uint32_t* taken, cudaStream_t s) {
    if (p.n) k_emitter_taken<<<blocks_for(p.n), kBlock, 0, s>>>(p, pos, cells, low, cnt, spacing, clear, taken);
}

void launch_emit(uint32_t total, const uint32_t* taken_ex, int3 cnt, float3 low, float spacing, float3 velocity,
                 uint32_t room, uint32_t first_id, float4* pos_out, float4* vel_out, uint32_t* ids_out, float* rho_out,
                 cudaStream_t s) {
    if (total && room)
        k_emit<<<blocks_for(total), kBlock, 0, s>>>(total, taken_ex, cnt, low, spacing, velocity, room, first_id, pos_out,
                                                    vel_out, ids_out, rho_out);
}

void launch_carry_movers(const Params& p, uint32_t k, const float4* start, const float4* vel, float elapsed, int3 low,
                         int3 span, uint32_t volume, uint32_t* lin, uint32_t* slot, uint32_t* table, uint32_t* tiles,
                         uint32_t* members, float4* start_out, float4* vel_out, float4* pos_out, cudaStream_t s) {
    if (!k) return;
    cudaMemsetAsync(table, 0, (size_t(volume) + 1) * 4, s);
    k_mover_cells<<<blocks_for(k), kBlock, 0, s>>>(p, k, start, vel, elapsed, low, span, lin, slot, table);
    launch_exclusive_scan(table, volume, tiles, s);
    k_mover_order<<<blocks_for(k), kBlock, 0, s>>>(k, lin, slot, table, members, start, vel, elapsed, start_out,
                                                   vel_out, pos_out, 0);
    k_mover_order<<<blocks_for(k), kBlock, 0, s>>>(k, lin, slot, table, members, start, vel, elapsed, start_out,
                                                   vel_out, pos_out, 1);
    g_launches.fetch_add(3, std::memory_order_relaxed);
}

void launch_in_boxes(uint32_t n, const float4* pos, const float3* boxes, uint32_t count, uint32_t* keep, cudaStream_t s) {
    if (n) k_in_boxes<<<blocks_for(n), kBlock, 0, s>>>(n, pos, boxes, count, keep);
}

void launch_gather_kept(uint32_t n, const uint32_t* keep, const uint32_t* at, const float4* pos, const float4* vel,
                        uint32_t* index, float* pv, cudaStream_t s) {
    if (n) k_gather_kept<<<blocks_for(n), kBlock, 0, s>>>(n, keep, at, pos, vel, index, pv);
}

void launch_scatter_velocities(uint32_t m, const uint32_t* index, const float* v3, float4* vel, cudaStream_t s) {
    if (m) k_scatter_velocities<<<blocks_for(m), kBlock, 0, s>>>(m, index, v3, vel);
}

void launch_domain_flags(const Params& p, const float4* pos, const int4* cells, float3 low, float3 high, int drain,
                         uint32_t* keep, cudaStream_t s) {
    if (p.n) k_domain_flags<<<blocks_for(p.n), kBlock, 0, s>>>(p, pos, cells, low, high, drain, keep);
}

void launch_compact(uint32_t n, const uint32_t* keep, const uint32_t* dest, const uint32_t* ids_in,
                    const float4* pos_in, const float4* vel_in, const float* rho_in, const int4* cells_in,
                    uint32_t* ids_out, float4* pos_out, float4* vel_out, float* rho_out, int4* cells_out,
                    const float2* warm_in, float2* warm_out, cudaStream_t s) {
    if (n)
        k_compact<<<blocks_for(n), kBlock, 0, s>>>(n, keep, dest, ids_in, pos_in, vel_in, rho_in, cells_in, ids_out,
                                                   pos_out, vel_out, rho_out, cells_out, warm_in, warm_out);
}

void launch_set_consts(const StepConsts& c, StepConsts* out, cudaStream_t s) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    k_set_consts<<<1, 1, 0, s>>>(c, out);
}

}  // namespace slf
